"""The phi-transform paths of SPH_MIXED plans that the size cases of
test_gpu_mixed.py do not reach, against the CPU oracle at the mixed form's
tolerance:

* the two-pass forward transform (nphi 1536) over more plane-fields than
  one batch of its scratch holds (64), so a second batch runs;
* an odd number of ring pairs (nlat/2 odd): tiles of 2, 4 or 8 ring pairs
  do not divide it, so both directions take the one-ring-pair kernels;
* a grid that is 8-byte but not 16-byte aligned (a view into a larger
  buffer): the forward transform's TMA and cp.async staging need 16-byte
  rows, so it takes the register-staged kernel; the inverse is unaffected.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import check, rel_l2, random_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-6


def _pair(lmax, nz, nlat, nphi):
    from redondito_b200 import sphp as S
    P = O.Plan(lmax, nz, nlat=nlat, nphi=nphi)
    G = S.Plan(lmax, nz, nlat=nlat, nphi=nphi, precision=S.SPH_MIXED)
    return P, G


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _round_trip(lmax, nz, nlat, nphi, grid_of=None, seed=0):
    from redondito_b200 import sphp as S
    P, G = _pair(lmax, nz, nlat, nphi)
    rng = np.random.default_rng(seed)
    spec = random_spec(P, rng, power=1.5, radial=False)
    grid_ref = P.sh_synthesis(spec)
    g = grid_of(G) if grid_of else G.new_grid()
    S.fftp2d_complex_to_real_xy(G, dev(spec), g)
    e_syn = rel_l2(host(g), grid_ref)
    g.copy_(dev(grid_ref))
    s = G.new_spec()
    S.fftp2d_real_to_complex_xy(G, g, s)
    e_ana = rel_l2(host(s), P.sh_analysis(grid_ref))
    S.plan_status(G)
    G.close()
    return e_syn, e_ana


def test_two_pass_forward_over_two_batches():
    e_syn, e_ana = _round_trip(511, 66, 768, 1536, seed=66)
    print(f"lmax 511, 66 planes: synthesis {e_syn:.2e} analysis {e_ana:.2e}")
    check(e_syn, TOL_MIXED, 'synthesis')
    check(e_ana, TOL_MIXED, 'analysis')


def test_odd_ring_pair_count():
    e_syn, e_ana = _round_trip(31, 5, 50, 96, seed=50)
    print(f"nlat 50: synthesis {e_syn:.2e} analysis {e_ana:.2e}")
    check(e_syn, TOL_MIXED, 'synthesis')
    check(e_ana, TOL_MIXED, 'analysis')


@pytest.mark.parametrize("lmax,nlat,nphi", [(63, 96, 192), (511, 768, 1536)])
def test_grid_not_16_byte_aligned(lmax, nlat, nphi):
    def offset_grid(G):
        n = G.nz * G.nphi * G.nlat
        flat = torch.empty(n + 1, dtype=torch.float64, device=G.device)
        g = flat[1:].view(G.nz, G.nphi, G.nlat)
        assert g.data_ptr() % 16 == 8
        return g

    e_syn, e_ana = _round_trip(lmax, 3, nlat, nphi, grid_of=offset_grid, seed=lmax)
    print(f"offset grid lmax {lmax}: synthesis {e_syn:.2e} analysis {e_ana:.2e}")
    check(e_syn, TOL_MIXED, 'synthesis')
    check(e_ana, TOL_MIXED, 'analysis')
