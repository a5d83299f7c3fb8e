"""SPH_MIXED plans (tensor-core Legendre contractions, fp32 phi FFTs) against
the CPU oracle on the same seeded inputs.  The mixed form splits every
operand into three bf16 pieces (about 24 significant bits) and accumulates
in fp32, so its transforms are held to relative L2 <= 1e-6 (TOL_MIXED),
the 3D transforms with FC-Gram continuation included; right-hand sides that
take radial derivatives are held to TOL_NL."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import check, rel_l2, random_spec

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
    check(e_syn, TOL_MIXED)
    check(e_ana, TOL_MIXED)


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
    check(max(e_syn), TOL_MIXED)
    check(max(e_ana), TOL_MIXED)


def test_mixed_full_angular_size():
    """lmax 511 on the 768 x 1536 grid (two planes): 256 rows per parity."""
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
    check(e_syn, TOL_MIXED)
    check(e_rt, 2 * TOL_MIXED)


def test_mixed_3d_vector_pair_with_continuation():
    from redondito_b200 import sphp as S
    P, G = _pair(63, 70, 96, 192, C=25, d=5)
    rng = np.random.default_rng(78)
    qst = [P.z_forward(random_spec(P, rng)) for _ in range(3)]
    for x in qst[1:]:
        x[:, 0] = 0
    ref_grids = P.qst_synthesis(*(P.z_inverse(x) for x in qst))
    g = [G.new_grid() for _ in range(3)]
    S.fftp3d_qst_to_vec(G, *(dev(x) for x in qst), *g)
    e_inv = [rel_l2(host(a), b) for a, b in zip(g, ref_grids)]
    ref = [P.z_forward(x) for x in P.qst_analysis(*ref_grids)]
    out = [G.new_spec() for _ in range(3)]
    S.fftp3d_vec_to_qst(G, *(dev(x) for x in ref_grids), *out)
    S.plan_status(G)
    e_fwd = [rel_l2(host(a), b) for a, b in zip(out, ref)]
    print(f"3D vector inverse {max(e_inv):.2e} forward {max(e_fwd):.2e}")
    check(max(e_inv), TOL_MIXED)
    check(max(e_fwd), TOL_MIXED)


def test_mixed_nl_rhs():
    """The NL step on a mixed plan (its continuation-feeding planes in FP64):
    the right-hand sides, which take radial derivatives of the analysed
    products, against the FP64 oracle within TOL_NL."""
    from redondito_b200 import sphp as S
    TOL_NL = 1e-5
    P, G = _pair(15, 64, 24, 48, C=25, d=5)
    P.bc_setup()
    S.setup_bc(G)
    rng = np.random.default_rng(3)
    Z = random_spec(P, rng, power=3.0)
    W = random_spec(P, rng, power=3.0)
    Z, phi, W = P.imposebc(Z, P.dlr(W))
    rz_ref, rf_ref, e_ref = P.nl_rhs(Z, W, phi, 1e-3)
    rz, rf = G.new_spec(), G.new_spec()
    e = S.nl_rhs(G, dev(Z), dev(W), dev(phi), 1e-3, rz, rf)
    S.plan_status(G)
    print(f"NL rhs_z {rel_l2(host(rz), rz_ref):.2e} rhs_phi {rel_l2(host(rf), rf_ref):.2e} energy {abs(e - e_ref) / e_ref:.2e}")
    check(abs(e - e_ref) / e_ref, TOL_MIXED)
    check(rel_l2(host(rz), rz_ref), TOL_NL)
    check(rel_l2(host(rf), rf_ref), TOL_NL)


def test_mixed_3d_pair_with_continuation():
    from redondito_b200 import sphp as S
    P, G = _pair(31, 64, 48, 96, C=25, d=5)
    rng = np.random.default_rng(77)
    spec = random_spec(P, rng)
    grid = P.sh_synthesis(spec)
    ref = P.forward_3d(grid)
    s = G.new_spec()
    S.fftp3d_real_to_complex(G, dev(grid), s)
    check(rel_l2(host(s), ref), TOL_MIXED)
    g = G.new_grid()
    S.fftp3d_complex_to_real(G, s, g)
    S.plan_status(G)
    check(rel_l2(host(g), P.inverse_3d(ref)), TOL_MIXED)


def test_mixed_zero_and_spike_inputs():
    """A zero field stays exactly zero; one large coefficient among small ones
    is resolved to the same relative accuracy (bf16 pieces need no scaling)."""
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
    check(rel_l2(host(g), grid_ref), TOL_MIXED)


@pytest.mark.parametrize("lmax,nz,nlat,nphi", [(63, 64, 96, 192), (127, 96, 192, 384), (31, 33, 48, 96),
                                             (31, 256, 48, 96)])
def test_3d_inverse_through_tiles_equals_the_composition(lmax, nz, nlat, nphi):
    """The mixed 3D inverses write the z inverse straight into the synthesis
    tiles (nz with a compile-time transform length; nz 33 takes the
    composition itself; nz 256 the 16 x 16 split in both paths): bit for bit
    the z inverse in place followed by the 2D synthesis, and the input is
    left unchanged."""
    from redondito_b200 import sphp as S
    P, G = _pair(lmax, nz, nlat, nphi, C=25, d=5)
    rng = np.random.default_rng(lmax + nz)
    fields = [dev(P.z_forward(random_spec(P, rng))) for _ in range(3)]
    fields[1][:, 0] = 0
    fields[2][:, 0] = 0
    x = fields[0].clone()
    g = G.new_grid()
    S.fftp3d_complex_to_real(G, x, g)
    if nz != 33:
        assert torch.equal(x, fields[0])
    y = fields[0].clone()
    S.fftp1d_complex_to_real_z(G, y)
    g2 = G.new_grid()
    S.fftp2d_complex_to_real_xy(G, y, g2)
    assert torch.equal(g, g2)
    q, s, t = (f.clone() for f in fields)
    v = [G.new_grid() for _ in range(3)]
    S.fftp3d_qst_to_vec(G, q, s, t, *v)
    qq, ss, tt = (f.clone() for f in fields)
    for f in (qq, ss, tt):
        S.fftp1d_complex_to_real_z(G, f)
    v2 = [G.new_grid() for _ in range(3)]
    S.fftp2d_qst_to_vec(G, qq, ss, tt, *v2)
    for a, b in zip(v, v2):
        assert torch.equal(a, b)
    S.plan_status(G)
    G.close()
