"""CUDA path vs the CPU oracle on identical seeded inputs (prueba_gpu.f90's
design: same entry point, CPU oracle against the device path).  FP64
transforms must agree to relative L2 <= 1e-12.  Radial derivatives are held
against the extended-precision operator (oracle/extended.py) within the
oracle's own error for the same field, at least 1e-12 (check_derivative);
the boundary solve runs on the extended-precision tables on both sides."""
import numpy as np
import pytest

from oracle import extended as X
from oracle import oracle as O
from tests._helpers import check, check_derivative, rel_l2, random_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# also for the outputs through the FC-Gram continuation (3D forward
# transforms), whose weights (up to 3.7e3) amplify the independent FP64
# rounding of the two sides: measured up to 8e-13
TOL = 1e-12


def _pair(lmax, nz, C=0, d=0, nlat=None, nphi=None, rint=0.35, rext=1.0):
    from redondito_b200 import sphp as S
    P = O.Plan(lmax, nz, nlat=nlat, nphi=nphi, C=C, d=d, rint=rint, rext=rext)
    G = S.Plan(lmax, nz, nlat=P.nlat, nphi=P.nphi, Cz=C, oz=d, rint=rint, rext=rext)
    return P, G


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


CASES_2D = [(15, 6, 24, 48), (31, 5, 48, 96), (63, 3, 96, 192), (7, 4, 12, 24)]


@pytest.mark.parametrize("lmax,nz,nlat,nphi", CASES_2D)
def test_sht_scalar(lmax, nz, nlat, nphi):
    from redondito_b200 import sphp as S
    P, G = _pair(lmax, nz, nlat=nlat, nphi=nphi)
    rng = np.random.default_rng(lmax)
    spec = random_spec(P, rng, radial=False)
    grid_ref = P.sh_synthesis(spec)
    g = G.new_grid()
    S.fftp2d_complex_to_real_xy(G, dev(spec), g)
    check(rel_l2(host(g), grid_ref), TOL)
    s = G.new_spec()
    S.fftp2d_real_to_complex_xy(G, dev(grid_ref), s)
    spec_ref = P.sh_analysis(grid_ref)
    check(rel_l2(host(s), spec_ref), TOL)
    check(rel_l2(host(s), spec), TOL)


@pytest.mark.parametrize("lmax,nz,nlat,nphi", CASES_2D[:3])
def test_sht_vector(lmax, nz, nlat, nphi):
    from redondito_b200 import sphp as S
    P, G = _pair(lmax, nz, nlat=nlat, nphi=nphi)
    rng = np.random.default_rng(100 + lmax)
    q, s, t = (random_spec(P, rng, radial=False) for _ in range(3))
    s[:, 0] = 0
    t[:, 0] = 0
    vr, vt, vp = P.qst_synthesis(q, s, t)
    out = [G.new_grid() for _ in range(3)]
    S.fftp2d_qst_to_vec(G, dev(q), dev(s), dev(t), *out)
    for a, b in zip(out, (vr, vt, vp)):
        check(rel_l2(host(a), b), TOL)
    qs = [G.new_spec() for _ in range(3)]
    S.fftp2d_vec_to_qst(G, dev(vr), dev(vt), dev(vp), *qs)
    ref = P.qst_analysis(vr, vt, vp)
    for a, b in zip(qs, ref):
        check(rel_l2(host(a), b), TOL)


@pytest.mark.parametrize("nz,C,d", [(16, 0, 0), (64, 25, 5), (33, 25, 5), (58, 25, 5), (256, 25, 5), (96, 25, 5)])
def test_z_transforms(nz, C, d):
    from redondito_b200 import sphp as S
    P, G = _pair(15, nz, C=C, d=d, nlat=24, nphi=48)
    rng = np.random.default_rng(nz)
    f = random_spec(P, rng)
    t = dev(f)
    S.fftp1d_real_to_complex_z(G, t)
    ref = P.z_forward(f)
    check(rel_l2(host(t), ref), TOL)
    S.fftp1d_complex_to_real_z(G, t)
    check(rel_l2(host(t), P.z_inverse(ref)), TOL)


@pytest.mark.parametrize("nz", [33, 58])
def test_config1_round_trip_and_derivative(nz):
    """lmax=31, 48 x 96, r in [0.35, 1]: synthesis -> analysis -> derivr(.,1,'r')."""
    from redondito_b200 import sphp as S
    P, G = _pair(31, nz, C=25, d=5, nlat=48, nphi=96)
    rng = np.random.default_rng(20261203 + 1)
    spec = random_spec(P, rng)
    grid_ref = P.sh_synthesis(spec)
    back_ref = P.sh_analysis(grid_ref)
    g = G.new_grid()
    s = G.new_spec()
    d = G.new_spec()
    S.fftp2d_complex_to_real_xy(G, dev(spec), g)
    S.fftp2d_real_to_complex_xy(G, g, s)
    S.derivr(G, s, d, 1, "r")
    check(rel_l2(host(g), grid_ref), TOL)
    check(rel_l2(host(s), back_ref), TOL)
    check_derivative(host(d), P, back_ref, 1, f"config 1 nz {nz}")


def test_3d_pair():
    from redondito_b200 import sphp as S
    P, G = _pair(31, 64, C=25, d=5, nlat=48, nphi=96)
    rng = np.random.default_rng(9)
    grid = P.sh_synthesis(random_spec(P, rng))
    ref = P.forward_3d(grid)
    s = G.new_spec()
    S.fftp3d_real_to_complex(G, dev(grid), s)
    check(rel_l2(host(s), ref), TOL)
    g = G.new_grid()
    back_ref = P.inverse_3d(ref)
    S.fftp3d_complex_to_real(G, dev(ref), g)
    check(rel_l2(host(g), back_ref), TOL)


@pytest.fixture(scope="module")
def pseudo():
    from redondito_b200 import sphp as S
    P, G = _pair(7, 128, C=25, d=5, rint=0.5, rext=1.5)
    rng = np.random.default_rng(77)
    a = random_spec(P, rng)
    return S, P, G, a


def test_derivr_ops(pseudo):
    S, P, G, a = pseudo
    for order in (1, 2, 3, 4):
        b = G.new_spec()
        S.derivr(G, dev(a), b, order, "r")
        check_derivative(host(b), P, a, order, "derivr")
    ak = P.z_forward(a)
    b = G.new_spec()
    S.derivr(G, dev(ak), b, 1, "k")
    check(rel_l2(host(b), P.derivr(ak, 1, "k")), TOL)
    b = G.new_spec()
    S.dlr(G, dev(a), b)
    check_derivative(host(b), P, a, "dlr", "dlr")


@pytest.mark.parametrize("nz", [33, 58, 64, 256])
def test_derivr_sizes(nz):
    """derivr orders 1-4 and dlr at radix-2/3 and generic lengths."""
    from redondito_b200 import sphp as S
    P, G = _pair(15, nz, C=25, d=5, nlat=24, nphi=48, rint=0.5, rext=1.5)
    a = random_spec(P, np.random.default_rng(nz + 1))
    for order in (1, 2, 3, 4):
        b = G.new_spec()
        S.derivr(G, dev(a), b, order, "r")
        check_derivative(host(b), P, a, order, f"nz {nz}")
    b = G.new_spec()
    S.dlr(G, dev(a), b)
    check_derivative(host(b), P, a, "dlr", f"nz {nz}")


def test_pointwise_ops(pseudo):
    S, P, G, a = pseudo
    b = G.new_spec()
    S.laplang(G, dev(a), b)
    assert rel_l2(host(b), P.laplang(a)) == 0.0
    S.multr(G, dev(a), b, -2)
    check(rel_l2(host(b), P.multr(a, -2)), 1e-15)
    c = G.new_spec()
    S.copy(G, dev(a), c)
    assert rel_l2(host(c), a) == 0.0
    y = P.derivr(a, 1)
    S.saxpby_c(G, c, dev(a), 2.0, dev(y), -3.0)
    check(rel_l2(host(c), P.saxpby_c(a, 2.0, y, -3.0)), 1e-15)
    f = dev(a)
    S.fc_filter(G, f, "r")
    check(rel_l2(host(f), P.fc_filter(a)), TOL)
    ak = P.z_forward(a)
    f = dev(ak)
    S.fc_filter(G, f, "k")
    check(rel_l2(host(f), P.fc_filter(ak, "k")), TOL)


def test_prodvec(pseudo):
    S, P, G, a = pseudo
    rng = np.random.default_rng(5)
    U = [rng.normal(size=P.grid_shape()) for _ in range(6)]
    ref = P.prodvec(U[:3], U[3:])
    out = [G.new_grid() for _ in range(3)]
    S.prodvec(G, *[dev(u) for u in U], *out)
    for o, r in zip(out, ref):
        assert rel_l2(host(o), r) == 0.0
    g = G.new_grid()
    S.saxpby_r(G, g, dev(U[0]), 0.5, dev(U[1]), 2.0)
    assert rel_l2(host(g), P.saxpby_r(U[0], 0.5, U[1], 2.0)) == 0.0


def test_boundary(pseudo):
    """invDl and v_imposebc(_fast) with no-slip walls against the oracle on
    the extended-precision boundary tables, which the CUDA path's long double
    setup reproduces to rounding (the comparison with the extended values
    themselves and with the oracle's own FP64 setup is in
    test_gpu_boundary_kinds.py)."""
    S, P, G, a = pseudo
    S.setup_bc(G)
    P.bc_setup(("noslip", "noslip"), tables=X.bc_tables(P, ("noslip", "noslip")))
    rng = np.random.default_rng(11)
    tor = random_spec(P, rng)
    phi = random_spec(P, rng)
    w = G.new_spec()
    S.invDl(G, dev(phi), w)
    check(rel_l2(host(w), P.invDl(phi)), TOL)
    t_ref, f_ref, w_ref = P.imposebc(tor, phi)
    T, F, W = dev(tor), dev(phi), G.new_spec()
    S.v_imposebc(G, T, F, W)
    assert rel_l2(host(T), t_ref) == 0.0
    check(rel_l2(host(W), w_ref), TOL)
    check(rel_l2(host(F), f_ref), TOL)
    t_ref, f_ref, w_ref = P.imposebc(tor, phi, fast=True)
    T, F, W = dev(tor), dev(phi), G.new_spec()
    S.v_imposebc_fast(G, T, F, W)
    check(rel_l2(host(W), w_ref), TOL)
    check(rel_l2(host(F), f_ref), TOL)


def test_nl_rhs_and_rk3():
    from redondito_b200 import sphp as S
    P, G = _pair(15, 64, C=25, d=5, nlat=24, nphi=48, rint=0.5, rext=1.5)
    P.bc_setup(("noslip", "noslip"), tables=X.bc_tables(P, ("noslip", "noslip")))
    S.setup_bc(G)
    rng = np.random.default_rng(3)
    Z = random_spec(P, rng, power=3.0)
    W = random_spec(P, rng, power=3.0)
    Z, phi, W = P.imposebc(Z, P.dlr(W))
    rz_ref, rf_ref, e_ref = P.nl_rhs(Z, W, phi, 1e-3)
    rz, rf = G.new_spec(), G.new_spec()
    e = S.nl_rhs(G, dev(Z), dev(W), dev(phi), 1e-3, rz, rf)
    check(abs(e - e_ref) / e_ref, 1e-12)
    check(rel_l2(host(rz), rz_ref), TOL)
    check(rel_l2(host(rf), rf_ref), TOL)
    Zr, Wr, Fr, e_ref = P.rk3_step(Z, W, phi, 1e-3, 1e-4)
    Zg, Wg, Fg = dev(Z), dev(W), dev(phi)
    e = S.rk3_step(G, Zg, Wg, Fg, 1e-3, 1e-4)
    check(abs(e - e_ref) / e_ref, 1e-12)
    check(rel_l2(host(Zg), Zr), TOL)
    check(rel_l2(host(Wg), Wr), TOL)
    check(rel_l2(host(Fg), Fr), TOL)


@pytest.mark.parametrize("lmax,nlat,nphi", [(255, 384, 768), (511, 768, 1536)])
def test_sht_full_angular_size(lmax, nlat, nphi):
    """The benchmark's angular sizes (compile-time 768/1536-point phi FFTs),
    scalar and vector, on two planes."""
    from redondito_b200 import sphp as S
    P, G = _pair(lmax, 2, nlat=nlat, nphi=nphi)
    rng = np.random.default_rng(lmax + 7)
    a = random_spec(P, rng, power=1.0, radial=False)
    g_ref = P.sh_synthesis(a)
    g = G.new_grid()
    S.fftp2d_complex_to_real_xy(G, dev(a), g)
    check(rel_l2(host(g), g_ref), TOL)
    s = G.new_spec()
    S.fftp2d_real_to_complex_xy(G, dev(g_ref), s)
    check(rel_l2(host(s), P.sh_analysis(g_ref)), TOL)
    q, sv, tv = a, random_spec(P, rng, power=1.0, radial=False), random_spec(P, rng, power=1.0, radial=False)
    sv[:, 0] = 0
    tv[:, 0] = 0
    v_ref = P.qst_synthesis(q, sv, tv)
    out = [G.new_grid() for _ in range(3)]
    S.fftp2d_qst_to_vec(G, dev(q), dev(sv), dev(tv), *out)
    for o, r in zip(out, v_ref):
        check(rel_l2(host(o), r), TOL)
    qs = [G.new_spec() for _ in range(3)]
    S.fftp2d_vec_to_qst(G, *[dev(x) for x in v_ref], *qs)
    for o, r in zip(qs, P.qst_analysis(*v_ref)):
        check(rel_l2(host(o), r), TOL)


def test_3d_vector_pair():
    """fftp3d_qst_to_vec / fftp3d_vec_to_qst equal the compositions of the
    2D vector transforms with the z transforms of q, s, t."""
    from redondito_b200 import sphp as S
    P, G = _pair(31, 64, C=25, d=5, nlat=48, nphi=96)
    rng = np.random.default_rng(21)
    qst = [P.z_forward(random_spec(P, rng)) for _ in range(3)]
    for x in qst[1:]:
        x[:, 0] = 0
    ref_grids = P.qst_synthesis(*(P.z_inverse(x) for x in qst))
    d = [dev(x) for x in qst]
    g = [G.new_grid() for _ in range(3)]
    S.fftp3d_qst_to_vec(G, *d, *g)
    for a, b in zip(g, ref_grids):
        check(rel_l2(host(a), b), TOL)
    ref = [P.z_forward(x) for x in P.qst_analysis(*ref_grids)]
    out = [G.new_spec() for _ in range(3)]
    S.fftp3d_vec_to_qst(G, *(dev(x) for x in ref_grids), *out)
    for a, b in zip(out, ref):
        check(rel_l2(host(a), b), TOL)
