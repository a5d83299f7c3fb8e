"""SPH_MIXED plans (tensor-core Legendre contractions, fp32 phi FFTs) against
the CPU oracle on the same seeded inputs.  The mixed form keeps about 22
significant bits per operand and accumulates in fp32, so its outputs are
held to relative L2 <= 1e-6 (TOL_MIXED); outputs that also pass through the
FP64 z transforms with FC-Gram continuation keep the same bound."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import rel_l2, random_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-6


def _pair(lmax, nz, nlat, nphi, C=0, d=0):
    from redondito_b200 import sphp as S
    P = O.Plan(lmax, nz, nlat=nlat, nphi=nphi, C=C, d=d)
    G = S.Plan(lmax, nz, nlat=nlat, nphi=nphi, Cz=C, oz=d, precision=S.SPH_MIXED)
    return P, G


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# (lmax, nz, nlat, nphi): small grids, a ragged plane block (nz = 70), the
# largest row blocks (lmax 255: 128 l per parity) and lmax 511 on 2 planes
CASES = [(7, 4, 12, 24), (15, 6, 24, 48), (31, 5, 48, 96), (63, 3, 96, 192), (127, 70, 192, 384),
         (255, 3, 384, 768)]


@pytest.mark.parametrize("lmax,nz,nlat,nphi", CASES)
def test_mixed_scalar(lmax, nz, nlat, nphi):
    from redondito_b200 import sphp as S
    P, G = _pair(lmax, nz, nlat, nphi)
    rng = np.random.default_rng(500 + lmax)
    spec = random_spec(P, rng, radial=False)
    grid_ref = P.sh_synthesis(spec)
    g = G.new_grid()
    S.fftp2d_complex_to_real_xy(G, dev(spec), g)
    e_syn = rel_l2(host(g), grid_ref)
    s = G.new_spec()
    S.fftp2d_real_to_complex_xy(G, dev(grid_ref), s)
    e_ana = rel_l2(host(s), P.sh_analysis(grid_ref))
    S.plan_status(G)
    print(f"lmax={lmax} synthesis {e_syn:.2e} analysis {e_ana:.2e}")
    assert e_syn < TOL_MIXED
    assert e_ana < TOL_MIXED


@pytest.mark.parametrize("lmax,nz,nlat,nphi", CASES[:4] + CASES[5:])
def test_mixed_vector(lmax, nz, nlat, nphi):
    from redondito_b200 import sphp as S
    P, G = _pair(lmax, nz, nlat, nphi)
    rng = np.random.default_rng(600 + lmax)
    q, s, t = (random_spec(P, rng, radial=False) for _ in range(3))
    s[:, 0] = 0
    t[:, 0] = 0
    ref = P.qst_synthesis(q, s, t)
    out = [G.new_grid() for _ in range(3)]
    S.fftp2d_qst_to_vec(G, dev(q), dev(s), dev(t), *out)
    e_syn = [rel_l2(host(a), b) for a, b in zip(out, ref)]
    qs = [G.new_spec() for _ in range(3)]
    S.fftp2d_vec_to_qst(G, *(dev(x) for x in ref), *qs)
    e_ana = [rel_l2(host(a), b) for a, b in zip(qs, P.qst_analysis(*ref))]
    S.plan_status(G)
    print(f"lmax={lmax} synthesis {max(e_syn):.2e} analysis {max(e_ana):.2e}")
    assert max(e_syn) < TOL_MIXED
    assert max(e_ana) < TOL_MIXED


def test_mixed_full_angular_size():
    """lmax 511 on the 768 x 1536 grid (two planes): the 256-row items."""
    from redondito_b200 import sphp as S
    P, G = _pair(511, 2, 768, 1536)
    rng = np.random.default_rng(511)
    spec = random_spec(P, rng, power=1.5, radial=False)
    grid_ref = P.sh_synthesis(spec)
    g = G.new_grid()
    S.fftp2d_complex_to_real_xy(G, dev(spec), g)
    s = G.new_spec()
    S.fftp2d_real_to_complex_xy(G, g, s)
    S.plan_status(G)
    e_syn = rel_l2(host(g), grid_ref)
    e_rt = rel_l2(host(s), spec)
    print(f"lmax=511 synthesis {e_syn:.2e} round trip {e_rt:.2e}")
    assert e_syn < TOL_MIXED
    assert e_rt < 2 * TOL_MIXED


def test_mixed_3d_pair_with_continuation():
    from redondito_b200 import sphp as S
    P, G = _pair(31, 64, 48, 96, C=25, d=5)
    rng = np.random.default_rng(77)
    spec = random_spec(P, rng)
    grid = P.sh_synthesis(spec)
    ref = P.forward_3d(grid)
    s = G.new_spec()
    S.fftp3d_real_to_complex(G, dev(grid), s)
    assert rel_l2(host(s), ref) < TOL_MIXED
    g = G.new_grid()
    S.fftp3d_complex_to_real(G, s, g)
    S.plan_status(G)
    assert rel_l2(host(g), P.inverse_3d(ref)) < TOL_MIXED


def test_mixed_zero_and_spike_inputs():
    """A zero field stays exactly zero; one large coefficient among small ones
    is resolved to the same relative accuracy (per-field power-of-two scale)."""
    from redondito_b200 import sphp as S
    P, G = _pair(31, 4, 48, 96)
    s = G.new_spec()
    S.fftp2d_real_to_complex_xy(G, G.new_grid(), s)
    assert float(s.abs().max()) == 0.0
    g = G.new_grid()
    S.fftp2d_complex_to_real_xy(G, G.new_spec(), g)
    assert float(g.abs().max()) == 0.0
    rng = np.random.default_rng(3)
    spec = random_spec(P, rng, radial=False)
    spec[:, 40] = 1e6
    grid_ref = P.sh_synthesis(spec)
    S.fftp2d_complex_to_real_xy(G, dev(spec), g)
    S.plan_status(G)
    assert rel_l2(host(g), grid_ref) < TOL_MIXED
