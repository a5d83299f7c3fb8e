"""The CUDA path against the CPU oracle at the benchmark's full sizes.

C3 (the benchmark workload): a scalar and a vector field at lmax 511 on the
768 x 1536 Gauss grid, nz 256 with FC-Gram C = 25, d = 5 -- the benchmark's
own seeded state (coefficients N(0,1)(l+1)^-2.5, real for m = 0, with 1% of
the (r, l, m) entries at amplitude 1e3 and random phase), in (lm, kz).  The
pair's inverse (fftp3d_complex_to_real, and z inverse + fftp2d_qst_to_vec for
the vector field) runs from that state and its forward
(fftp3d_real_to_complex, and fftp2d_vec_to_qst + z forward) from the
oracle's grids, so each direction is compared on identical inputs.  The
FP64 form is held to the required relative L2 of 1e-12 per output, the
mixed form to 1e-6 per output.

C2: the vector nonlinear step at lmax 255, 384 x 768, nz 128, with the
no-slip rows imposed by v_imposebc (src/boundary/vboundary.f90:59-87):
the right-hand sides and the FP64 energy, and one RK3 step.  The oracle runs
here on the boundary matrices evaluated in long double (oracle/extended.py),
as the CUDA path builds them; the boundary solve is also compared with the
extended-precision values themselves.

The oracle runs on every host core (about a minute in all on 16 cores).
"""
import os
import sys

import numpy as np
import pytest

from oracle import extended as X
from oracle import oracle as O
from tests._helpers import check, random_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-12
TOL_MIXED = 1e-6
# right-hand sides of the NL step take radial derivatives of analysed products
TOL_NL_MIXED = 1e-5


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def rel_dev(a, b):
    """Relative L2 of a (CUDA tensor) against b (numpy), computed on the device."""
    bd = dev(b)
    r = float((torch.linalg.vector_norm(a - bd) / torch.linalg.vector_norm(bd)).item())
    del bd
    return r


@pytest.fixture(scope="module")
def c3():
    """The benchmark's seeded C3 state and the oracle's pair on it."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    from redondito_b200 import sphp as S
    W = bench.CASES["c3"]
    Pd = S.Plan(W["lmax"], W["nz"], nlat=W["nlat"], nphi=W["nphi"], Cz=W["Cz"], oz=W["oz"],
                rint=W["rint"], rext=W["rext"])
    gen = torch.Generator(device=Pd.device)
    gen.manual_seed(bench.SEED)
    st = bench.make_state(S, Pd, torch, gen)
    spec = [x.cpu().numpy() for x in st]
    del st
    P = O.Plan(W["lmax"], W["nz"], nlat=W["nlat"], nphi=W["nphi"], C=W["Cz"], d=W["oz"],
               rint=W["rint"], rext=W["rext"])
    grids = [P.inverse_3d(spec[0])]
    grids += list(P.qst_synthesis(*(P.z_inverse(x) for x in spec[1:])))
    fwd = [P.forward_3d(grids[0])]
    fwd += [P.z_forward(x) for x in P.qst_analysis(*grids[1:])]
    yield dict(W=W, Pd=Pd, spec=spec, grids=grids, fwd=fwd)
    Pd.close()


def _run_pair(S, G, c):
    """The pair on plan G: inverse from the state, forward from the oracle's grids."""
    a, q, s, t = (dev(x) for x in c["spec"])
    g = [G.new_grid() for _ in range(4)]
    S.fftp3d_complex_to_real(G, a, g[0])
    S.fftp3d_qst_to_vec(G, q, s, t, g[1], g[2], g[3])
    del a, q, s, t
    inv = [rel_dev(x, r) for x, r in zip(g, c["grids"])]
    del g
    gin = [dev(x) for x in c["grids"]]
    out = [G.new_spec() for _ in range(4)]
    S.fftp3d_real_to_complex(G, gin[0], out[0])
    S.fftp3d_vec_to_qst(G, gin[1], gin[2], gin[3], out[1], out[2], out[3])
    del gin
    fwd = [rel_dev(x, r) for x, r in zip(out, c["fwd"])]
    return inv, fwd


NAMES_INV = ("grid scalar", "grid v_r", "grid v_theta", "grid v_phi")
NAMES_FWD = ("spec scalar", "Q", "S", "T")


def test_c3_fp64_pair_against_oracle(c3):
    from redondito_b200 import sphp as S
    inv, fwd = _run_pair(S, c3["Pd"], c3)
    for name, e in zip(NAMES_INV + NAMES_FWD, inv + fwd):
        check(e, TOL, "C3 FP64 " + name)


def test_c3_mixed_pair_against_oracle(c3):
    from redondito_b200 import sphp as S
    W = c3["W"]
    G = S.Plan(W["lmax"], W["nz"], nlat=W["nlat"], nphi=W["nphi"], Cz=W["Cz"], oz=W["oz"],
               rint=W["rint"], rext=W["rext"], precision=S.SPH_MIXED)
    inv, fwd = _run_pair(S, G, c3)
    S.plan_status(G)
    G.close()
    for name, e in zip(NAMES_INV + NAMES_FWD, inv + fwd):
        check(e, TOL_MIXED, "C3 mixed " + name)


@pytest.fixture(scope="module")
def c2():
    """C2: Z, W ~ N(0,1)(l+1)^-3 times a smooth radial profile, phi = D_l W,
    the no-slip rows imposed by the oracle's v_imposebc on the
    extended-precision boundary tables (the CUDA path builds its matrices in
    long double too; the reference's FP64 setup is compared separately)."""
    lmax, nz, nlat, nphi = 255, 128, 384, 768
    P = O.Plan(lmax, nz, nlat=nlat, nphi=nphi, C=25, d=5, rint=0.35, rext=1.0)
    P.bc_setup(("noslip", "noslip"), tables=X.bc_tables(P, ("noslip", "noslip")))
    rng = np.random.default_rng(20261203 + 2)
    Z0 = random_spec(P, rng, power=3.0)
    W0 = random_spec(P, rng, power=3.0)
    Z, phi, W = P.imposebc(Z0, P.dlr(W0))
    rz, rf, e = P.nl_rhs(Z, W, phi, 1e-3)
    return dict(P=P, raw=(Z0, P.dlr(W0)), state=(Z, W, phi), nl=(rz, rf, e),
                exact=X.imposebc_rows(P, ("noslip", "noslip"), P.dlr(W0)))


def _gpu_plan(prec):
    from redondito_b200 import sphp as S
    G = S.Plan(255, 128, nlat=384, nphi=768, Cz=25, oz=5, rint=0.35, rext=1.0, precision=prec)
    S.setup_bc(G)
    return G


def test_c2_imposebc_fp64(c2):
    from redondito_b200 import sphp as S
    G = _gpu_plan(S.SPH_FP64)
    T, F = (dev(x) for x in c2["raw"])
    Wg = G.new_spec()
    S.v_imposebc(G, T, F, Wg)
    Z, W, phi = c2["state"]
    check(rel_dev(T, Z), TOL, "C2 tor")
    check(rel_dev(Wg, W), TOL, "C2 pol")
    check(rel_dev(F, phi), TOL, "C2 phi")
    n = c2["P"].N
    w_x, f_x = c2["exact"]
    check(X.rel_l2(Wg.cpu().numpy()[:n], w_x), 1e-14, "C2 pol vs extended")
    check(X.rel_l2(F.cpu().numpy()[:n], f_x), TOL, "C2 phi vs extended")
    G.close()


def test_c2_nl_step_fp64(c2):
    from redondito_b200 import sphp as S
    G = _gpu_plan(S.SPH_FP64)
    Z, W, phi = c2["state"]
    rz_ref, rf_ref, e_ref = c2["nl"]
    rz, rf = G.new_spec(), G.new_spec()
    e = S.nl_rhs(G, dev(Z), dev(W), dev(phi), 1e-3, rz, rf)
    check(abs(e - e_ref) / e_ref, TOL, "C2 energy")
    check(rel_dev(rz, rz_ref), TOL, "C2 rhs_z")
    check(rel_dev(rf, rf_ref), TOL, "C2 rhs_phi")
    G.close()


def test_c2_rk3_step_fp64(c2):
    from redondito_b200 import sphp as S
    P = c2["P"]
    Z, W, phi = c2["state"]
    Zr, Wr, Fr, e_ref = P.rk3_step(Z, W, phi, 1e-3, 1e-4)
    G = _gpu_plan(S.SPH_FP64)
    Zg, Wg, Fg = dev(Z), dev(W), dev(phi)
    e = S.rk3_step(G, Zg, Wg, Fg, 1e-3, 1e-4)
    check(abs(e - e_ref) / e_ref, TOL, "C2 RK3 energy")
    check(rel_dev(Zg, Zr), TOL, "C2 RK3 Z")
    check(rel_dev(Wg, Wr), TOL, "C2 RK3 W")
    check(rel_dev(Fg, Fr), TOL, "C2 RK3 phi")
    G.close()


def test_c2_nl_step_mixed(c2):
    from redondito_b200 import sphp as S
    G = _gpu_plan(S.SPH_MIXED)
    Z, W, phi = c2["state"]
    rz_ref, rf_ref, e_ref = c2["nl"]
    rz, rf = G.new_spec(), G.new_spec()
    e = S.nl_rhs(G, dev(Z), dev(W), dev(phi), 1e-3, rz, rf)
    S.plan_status(G)
    check(abs(e - e_ref) / e_ref, TOL_MIXED, "C2 mixed energy")
    check(rel_dev(rz, rz_ref), TOL_NL_MIXED, "C2 mixed rhs_z")
    check(rel_dev(rf, rf_ref), TOL_NL_MIXED, "C2 mixed rhs_phi")
    G.close()
