"""Single-precision entry points (the arrays of a GSINGLE_PRECISION build of
the reference, src/sphp/fprecision_mod.F90:13-18) on SPH_MIXED plans,
against the CPU oracle in FP64 on the same inputs (the float input widened):
the mixed form's bound (1e-6) plus the rounding of the float arrays, 2e-6.

Sizes: lmax 63 (three-step phi kernels on float grids by TMA), lmax 511
(the two-pass forward and the three-step inverse at nphi 1536), and nlat 50
(25 ring pairs: the register-staged kernels)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import check, random_spec, rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 2e-6


def f32(x):
    x = np.ascontiguousarray(x)
    return torch.from_numpy(x.astype(np.complex64 if np.iscomplexobj(x) else np.float32)).cuda()


def host64(t):
    torch.cuda.synchronize()
    x = t.cpu().numpy()
    return x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)


def widened(x):
    """the float-rounded input, back in FP64 (what the oracle sees)"""
    return host64(f32(x))


def _pair(lmax, nz, nlat, nphi, C=25, d=5):
    from redondito_b200 import sphp as S
    P = O.Plan(lmax, nz, nlat=nlat, nphi=nphi, C=C, d=d, rint=0.5, rext=1.5)
    G = S.Plan(lmax, nz, nlat=nlat, nphi=nphi, Cz=C, oz=d, rint=0.5, rext=1.5, precision=S.SPH_MIXED)
    return S, P, G


@pytest.mark.parametrize("lmax,nz,nlat,nphi", [(63, 64, 96, 192), (511, 32, 768, 1536), (31, 32, 50, 96)])
def test_3d_scalar_and_vector_pairs(lmax, nz, nlat, nphi):
    S, P, G = _pair(lmax, nz, nlat, nphi)
    rng = np.random.default_rng(lmax + nlat)
    spec = widened(P.z_forward(random_spec(P, rng)))
    # inverse from the float spectra; the input is preserved
    sf = f32(spec)
    s0 = sf.clone()
    g = G.new_grid32()
    S.fftp3d_complex_to_real_f32(G, sf, g)
    assert torch.equal(sf, s0)
    check(rel_l2(host64(g), P.inverse_3d(spec)), TOL, f"3D inverse lmax {lmax}")
    # forward from a float grid
    grid = widened(P.inverse_3d(spec))
    out = G.new_spec32()
    S.fftp3d_real_to_complex_f32(G, f32(grid), out)
    check(rel_l2(host64(out), P.forward_3d(grid)), TOL, f"3D forward lmax {lmax}")
    # vector
    qst = [widened(P.z_forward(random_spec(P, rng))) for _ in range(3)]
    for x in qst[1:]:
        x[:, 0] = 0
    g3 = [G.new_grid32() for _ in range(3)]
    S.fftp3d_qst_to_vec_f32(G, *(f32(x) for x in qst), *g3)
    ref = P.qst_synthesis(*(P.z_inverse(x) for x in qst))
    for a, b, name in zip(g3, ref, ("vr", "vt", "vp")):
        check(rel_l2(host64(a), b), TOL, f"3D qst_to_vec {name} lmax {lmax}")
    grids = [widened(x) for x in ref]
    o3 = [G.new_spec32() for _ in range(3)]
    S.fftp3d_vec_to_qst_f32(G, *(f32(x) for x in grids), *o3)
    ref = [P.z_forward(x) for x in P.qst_analysis(*grids)]
    for a, b, name in zip(o3, ref, "QST"):
        check(rel_l2(host64(a), b), TOL, f"3D vec_to_qst {name} lmax {lmax}")
    S.plan_status(G)
    G.close()


def test_2d_and_z_transforms():
    S, P, G = _pair(63, 64, 96, 192)
    rng = np.random.default_rng(3)
    spec = widened(random_spec(P, rng))
    g = G.new_grid32()
    S.fftp2d_complex_to_real_xy_f32(G, f32(spec), g)
    check(rel_l2(host64(g), P.sh_synthesis(spec)), TOL, "2D synthesis")
    grid = widened(P.sh_synthesis(spec))
    s = G.new_spec32()
    S.fftp2d_real_to_complex_xy_f32(G, f32(grid), s)
    check(rel_l2(host64(s), P.sh_analysis(grid)), TOL, "2D analysis")
    t = f32(spec)
    S.fftp1d_real_to_complex_z_f32(G, t)
    zf = P.z_forward(spec)
    check(rel_l2(host64(t), zf), TOL, "z forward")
    t = f32(zf)
    S.fftp1d_complex_to_real_z_f32(G, t)
    check(rel_l2(host64(t), P.z_inverse(widened(zf))), TOL, "z inverse")
    S.plan_status(G)
    G.close()


def test_radial_operators():
    S, P, G = _pair(15, 64, 24, 48)
    rng = np.random.default_rng(5)
    a = widened(random_spec(P, rng, power=3.0))
    n = P.N
    for order in (1, 2):
        b = G.new_spec32()
        S.derivr_f32(G, f32(a), b, order)
        check(rel_l2(host64(b)[:n], P.derivr(a, order)[:n]), TOL, f"derivr order {order}")
    b = G.new_spec32()
    S.dlr_f32(G, f32(a), b)
    check(rel_l2(host64(b)[:n], P.dlr(a)[:n]), TOL, "dlr")
    x = f32(a)
    S.fc_filter_f32(G, x, "r")
    check(rel_l2(host64(x), P.fc_filter(a)), TOL, "fc_filter")
    ak = widened(P.z_forward(a))
    b = G.new_spec32()
    S.derivr_f32(G, f32(ak), b, 1, "k")
    check(rel_l2(host64(b), P.derivr(ak, 1, "k")), TOL, "derivr in k")
    G.close()


def test_fp64_plans_are_refused():
    from redondito_b200 import sphp as S
    G = S.Plan(15, 64, nlat=24, nphi=48, Cz=25, oz=5, rint=0.5, rext=1.5)
    with pytest.raises(S.SphError):
        S.fftp3d_real_to_complex_f32(G, G.new_grid32(), G.new_spec32())
    G.close()


def test_pointwise_operators():
    """Computed in FP64 from the float inputs: within float rounding of the
    oracle on the widened inputs."""
    S, P, G = _pair(15, 64, 24, 48)
    rng = np.random.default_rng(8)
    a, y = widened(random_spec(P, rng)), widened(random_spec(P, rng))
    b = G.new_spec32()
    S.laplang_f32(G, f32(a), b)
    check(rel_l2(host64(b), P.laplang(a)), 1e-7, "laplang")
    S.multr_f32(G, f32(a), b, -2)
    check(rel_l2(host64(b), P.multr(a, -2)), 1e-7, "multr")
    z = G.new_spec32()
    S.saxpby_c_f32(G, z, f32(a), 2.0, f32(y), -3.0)
    check(rel_l2(host64(z), P.saxpby_c(a, 2.0, y, -3.0)), 1e-7, "saxpby_c")
    S.copy_f32(G, f32(a), b)
    assert rel_l2(host64(b), a) == 0.0
    x = f32(a)
    S.dirichlet_f32(G, x)
    check(rel_l2(host64(x), P.dirichlet(a)), 1e-7, "dirichlet")
    g = [widened(P.sh_synthesis(random_spec(P, rng))) for _ in range(6)]
    c = [G.new_grid32() for _ in range(3)]
    S.prodvec_f32(G, *(f32(v) for v in g), *c)
    for u, v, name in zip(c, P.prodvec(g[:3], g[3:]), ("r", "t", "p")):
        check(rel_l2(host64(u), v), 1e-7, f"prodvec {name}")
    zr = G.new_grid32()
    S.saxpby_r_f32(G, zr, f32(g[0]), 0.5, f32(g[1]), 2.0)
    check(rel_l2(host64(zr), P.saxpby_r(g[0], 0.5, g[1], 2.0)), 1e-7, "saxpby_r")
    G.close()


def test_boundary_and_nl_step_match_the_fp64_arrays():
    """The boundary solve, the NL step and RK3 on float arrays run the FP64
    routines on widened copies: their outputs equal the FP64-array calls on
    the same (widened) inputs to float rounding."""
    S, P, G = _pair(15, 64, 24, 48)
    S.setup_bc(G)
    rng = np.random.default_rng(9)
    Z = widened(random_spec(P, rng, power=3.0))
    W = widened(random_spec(P, rng, power=3.0))
    phi = widened(P.dlr(W))

    def d64(x):
        return torch.from_numpy(np.ascontiguousarray(x)).cuda()

    w32, w64 = G.new_spec32(), G.new_spec()
    S.invDl_f32(G, f32(phi), w32)
    S.invDl(G, d64(phi), w64)
    check(rel_l2(host64(w32), host64(w64)), 1e-7, "invDl")
    for fast in (False, True):
        t32, f32_, p32 = f32(Z), f32(phi), G.new_spec32()
        t64, f64_, p64 = d64(Z), d64(phi), G.new_spec()
        (S.v_imposebc_fast_f32 if fast else S.v_imposebc_f32)(G, t32, f32_, p32)
        (S.v_imposebc_fast if fast else S.v_imposebc)(G, t64, f64_, p64)
        for a, b, name in ((t32, t64, "tor"), (f32_, f64_, "phi"), (p32, p64, "pol")):
            check(rel_l2(host64(a), host64(b)), 1e-7, f"imposebc fast={fast} {name}")
    Zs, Ws, Fs = (widened(host64(x)) for x in (t64, p64, f64_))
    rz32, rf32, rz64, rf64 = G.new_spec32(), G.new_spec32(), G.new_spec(), G.new_spec()
    e32 = S.nl_rhs_f32(G, f32(Zs), f32(Ws), f32(Fs), 1e-3, rz32, rf32)
    e64 = S.nl_rhs(G, d64(Zs), d64(Ws), d64(Fs), 1e-3, rz64, rf64)
    assert abs(e32 - e64) <= 1e-12 * abs(e64)  # the energy sum is reduced with atomics
    check(rel_l2(host64(rz32), host64(rz64)), 1e-7, "rhs_z")
    check(rel_l2(host64(rf32), host64(rf64)), 1e-7, "rhs_phi")
    a32 = [f32(x) for x in (Zs, Ws, Fs)]
    a64 = [d64(x) for x in (Zs, Ws, Fs)]
    S.rk3_step_f32(G, *a32, 1e-3, 1e-4)
    S.rk3_step(G, *a64, 1e-3, 1e-4)
    for a, b, name in zip(a32, a64, ("Z", "W", "phi")):
        check(rel_l2(host64(a), host64(b)), 1e-7, f"RK3 {name}")
    S.plan_status(G)
    G.close()
