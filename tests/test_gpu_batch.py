"""Batches of independent problems (sph_batch_*): one CUDA graph with the
Legendre contractions of every problem in one grouped launch per direction.
Every output must equal, bit for bit, the same work done by the single-plan
entry points (the grouped launches run the same arithmetic per work unit),
and the FP64 batch must match the CPU oracle like the single-plan path."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import check, check_derivative, rel_l2, random_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12

# (lmax, nz, nfields): the C4 ensemble's shapes at small sizes (nlat = 3(lmax+1)/2, nphi = 2 nlat)
PROBLEMS = [(15, 32, 1), (31, 64, 3), (31, 32, 2), (63, 96, 1), (15, 64, 2), (63, 32, 3)]


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _problem_inputs(lmax, nz, nf, seed):
    nlat = 3 * (lmax + 1) // 2
    P = O.Plan(lmax, nz, nlat=nlat, nphi=2 * nlat, C=25, d=5)
    rng = np.random.default_rng(seed)
    return P, [P.z_forward(random_spec(P, rng)) for _ in range(nf)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_plan_calls(precision):
    from redondito_b200 import sphp as S
    prec = S.SPH_FP64 if precision == "fp64" else S.SPH_MIXED
    plans, inputs, orcs = [], [], []
    for i, (lmax, nz, nf) in enumerate(PROBLEMS):
        P, xs = _problem_inputs(lmax, nz, nf, 40 + i)
        orcs.append(P)
        plans.append(S.Plan(lmax, nz, nlat=P.nlat, nphi=P.nphi, Cz=25, oz=5, precision=prec))
        inputs.append(xs)
    B = S.Batch(plans, [len(x) for x in inputs])
    for p, xs in enumerate(inputs):
        for f, x in enumerate(xs):
            B.spec[p][f].copy_(dev(x))
    torch.cuda.synchronize()
    B.run()
    B.status()
    for p, (G, xs) in enumerate(zip(plans, inputs)):
        for f, x in enumerate(xs):
            s = dev(x)
            d = G.new_spec()
            g = G.new_grid()
            S.fftp1d_complex_to_real_z(G, s)
            S.derivr(G, s, d, 1, "r")
            S.fftp2d_complex_to_real_xy(G, s, g)
            out = G.new_spec()
            S.fftp3d_real_to_complex(G, g, out)
            torch.cuda.synchronize()
            assert torch.equal(B.grid[p][f], g), (p, f)
            assert torch.equal(B.dspec[p][f], d), (p, f)
            assert torch.equal(B.spec[p][f], out), (p, f)
            if precision == "fp64":
                P = orcs[p]
                sr = P.z_inverse(x)
                check(rel_l2(host(s), sr), TOL, "z inverse")
                check(rel_l2(host(g), P.sh_synthesis(sr)), TOL, "synthesis")
                # the derivative of the same (device) input on both sides
                check_derivative(host(d), P, host(s), 1, f"problem {p}")
                check(rel_l2(host(out), P.forward_3d(P.sh_synthesis(sr))), TOL, "3D forward")


def test_batch_replays():
    """A second run of the same graph on new inputs gives the new answers."""
    from redondito_b200 import sphp as S
    P, xs = _problem_inputs(31, 64, 2, 7)
    G = S.Plan(31, 64, nlat=P.nlat, nphi=P.nphi, Cz=25, oz=5, precision=S.SPH_MIXED)
    B = S.Batch([G], [2])
    for rep in range(2):
        ys = [x * (rep + 1.5) for x in xs]
        for f, y in enumerate(ys):
            B.spec[0][f].copy_(dev(y))
        torch.cuda.synchronize()
        B.run()
        B.status()
        for f, y in enumerate(ys):
            ref = P.sh_synthesis(P.z_inverse(y))
            check(rel_l2(host(B.grid[0][f]), ref), 1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tile_shapes_do_not_change_results(precision):
    from redondito_b200 import sphp as S
    prec = S.SPH_FP64 if precision == "fp64" else S.SPH_MIXED
    P, xs = _problem_inputs(63, 96, 1, 11)
    G = S.Plan(63, 96, nlat=P.nlat, nphi=P.nphi, Cz=25, oz=5, precision=prec)

    def run():
        s = dev(xs[0])
        g = G.new_grid()
        out = G.new_spec()
        S.fftp3d_complex_to_real(G, s, g)
        S.fftp3d_real_to_complex(G, g, out)
        return host(g), host(out)

    g0, o0 = run()
    S.set_tiles(G, 64 if prec else 0, 2, 16)
    g1, o1 = run()
    S.set_tiles(G, 32 if prec else 0, 4, 32)
    g2, o2 = run()
    # FP64: the built-in shape takes the cluster forward phi kernel, the set
    # ring pairs the single-CTA kernels, whose FFTs factor the length
    # differently (rounding differs; the continuation of the forward 3D
    # transform amplifies it); mixed: the MMA rows change the fp32 sums
    tol = 1e-12 if precision == "fp64" else 1e-9
    for g, o in ((g1, o1), (g2, o2)):
        check(rel_l2(g, g0), tol)
        check(rel_l2(o, o0), tol)
    with pytest.raises(S.SphError):
        S.set_tiles(G, 48, 0, 0)
    with pytest.raises(S.SphError):
        S.set_tiles(G, 0, 3, 0)


def test_batch_refuses_a_plan_twice():
    """A plan's per-field scratch serves one problem: the same plan for two
    problems of a batch would race on it, so sph_batch_create refuses it."""
    import ctypes
    from redondito_b200 import sphp as S
    G = S.Plan(15, 32, nlat=24, nphi=48, Cz=25, oz=5)
    bufs = [G.new_spec(), G.new_grid(), G.new_spec(), G.new_spec(), G.new_grid(), G.new_spec()]
    ph = (ctypes.c_void_p * 2)(G.h.value, G.h.value)
    nf = (ctypes.c_int * 2)(1, 1)
    arr = lambda a, b: (ctypes.c_void_p * 2)(a.data_ptr(), b.data_ptr())
    h = ctypes.c_void_p()
    rc = S.lib().sph_batch_create(ctypes.byref(h), 2, ph, nf, arr(bufs[0], bufs[3]), arr(bufs[1], bufs[4]),
                                  arr(bufs[2], bufs[5]))
    assert rc == 1 and not h.value  # SPH_EINVAL
    G2 = G.clone()
    ph2 = (ctypes.c_void_p * 2)(G.h.value, G2.h.value)
    rc = S.lib().sph_batch_create(ctypes.byref(h), 2, ph2, nf, arr(bufs[0], bufs[3]), arr(bufs[1], bufs[4]),
                                  arr(bufs[2], bufs[5]))
    assert rc == 0  # two plans (a clone has scratch of its own)
    S.lib().sph_batch_destroy(h)
    G2.close()
    G.close()
