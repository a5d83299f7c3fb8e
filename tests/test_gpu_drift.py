"""Error growth over repeated use of the transforms.

Round trips: the 3D inverse then forward transform of one state, 100 times.
The mixed form's Legendre contractions accumulate in fp32 on the tensor
cores, which truncate the aligned sum of every MMA toward zero: each trip
scales the state by about (1 - 4e-7) and adds an orthogonal error of about
1.3e-7, both systematic, so the error grows linearly with the number of
trips, not as its square root.  Bounds: after n trips the relative error is
below n x 6e-7 and its component along the state (a shrink) below n x 5e-7
in magnitude; the FP64 form stays below 2e-11 after 100 trips.

A time-stepping run does not compound it: its state stays FP64 in spectral
space and the transforms only evaluate the nonlinear term, so 20 RK3 steps
on a mixed plan stay within 3e-7 of the same steps on an FP64 plan, and
the difference grows at most linearly."""
import numpy as np
import pytest

from tests._helpers import check

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _state(P, seed, power=2.5):
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    ell = P.ell.cuda().double()
    emm = P.emm.cuda()
    amp = (ell + 1.0) ** -power
    re = torch.randn((P.nz, P.nlm), generator=gen, device="cuda", dtype=torch.float64)
    im = torch.randn((P.nz, P.nlm), generator=gen, device="cuda", dtype=torch.float64)
    x = torch.complex(re * amp, im * amp)
    x[:, emm == 0] = x[:, emm == 0].real.to(torch.complex128)
    return x.contiguous()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_round_trip_drift(precision):
    from redondito_b200 import sphp as S
    prec = S.SPH_MIXED if precision == "mixed" else S.SPH_FP64
    P = S.Plan(255, 64, nlat=384, nphi=768, Cz=25, oz=5, rint=0.35, rext=1.0, precision=prec)
    x = _state(P, 5)
    S.fftp1d_real_to_complex_z(P, x)
    x0 = x.clone()
    n0 = torch.linalg.vector_norm(x0)
    g = P.new_grid()
    rows = []
    for n in range(1, 101):
        S.fftp3d_complex_to_real(P, x, g)
        S.fftp3d_real_to_complex(P, g, x)
        if n in (1, 10, 25, 50, 100):
            d = x - x0
            rel = float(torch.linalg.vector_norm(d) / n0)
            c = float(torch.sum(d.conj() * x0).real / n0 ** 2)
            rows.append((n, rel, c))
    S.plan_status(P)
    P.close()
    for n, rel, c in rows:
        print(f"{precision} after {n} trips: relative error {rel:.3e}, along the state {c:+.3e}")
        if precision == "mixed":
            check(rel, n * 6e-7, f"mixed error after {n} trips")
            check(abs(c), n * 5e-7, f"mixed scaling after {n} trips")
        else:
            check(rel, 2e-11, f"fp64 error after {n} trips")


def test_rk3_run_does_not_compound():
    """20 RK3 steps on a mixed and an FP64 plan from the same state: the
    difference after 20 steps stays below 3e-7 and at most 2.5 times the
    difference after 10 (linear growth at most, no compounding)."""
    from redondito_b200 import sphp as S
    out = {}
    for name, prec in (("fp64", S.SPH_FP64), ("mixed", S.SPH_MIXED)):
        G = S.Plan(63, 64, nlat=96, nphi=192, Cz=25, oz=5, rint=0.5, rext=1.5, precision=prec)
        S.setup_bc(G)
        Z, W = _state(G, 11, 3.0), _state(G, 12, 3.0)
        F = G.new_spec()
        S.dlr(G, W, F)
        S.v_imposebc(G, Z, F, W)
        snaps = []
        for n in range(1, 21):
            S.rk3_step(G, Z, W, F, 1e-3, 1e-4, energy=False)
            if n in (10, 20):
                snaps.append((Z.clone(), W.clone(), F.clone()))
        S.plan_status(G)
        out[name] = snaps
        G.close()
    for i, name in enumerate(("Z", "W", "phi")):
        d = [float(torch.linalg.vector_norm(out["mixed"][j][i] - out["fp64"][j][i]) /
                   torch.linalg.vector_norm(out["fp64"][j][i])) for j in range(2)]
        print(f"RK3 mixed vs FP64, {name}: after 10 steps {d[0]:.3e}, after 20 steps {d[1]:.3e}")
        check(d[1], 3e-7, f"20 RK3 steps, mixed vs FP64, {name}")
        # at most linear growth (with an absolute allowance for differences
        # that start near zero, as phi's does after the first imposebc)
        check(d[1] - 2.5 * d[0], 2e-8, f"growth from 10 to 20 steps, {name}")
