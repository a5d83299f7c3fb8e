"""Oracle vs the known answers of the reference's prueba_vec.f90 (vector QST).

Convention (prueba_vec.f90:5-7): v = Q Y r + S r grad Y - T r x grad Y,
v_th = dS/dth + (1/sin th) dT/dph, v_ph = (1/sin th) dS/dph - dT/dth.
Reference errors: 1e-15 .. 6e-14 analysis, 1e-15 .. 1e-14 synthesis,
8e-13 for the sin^15 toroidal case, 3e-14 .. 9e-14 round trip (LEEME.md:42).
"""
import numpy as np
import pytest

from oracle import oracle as O

LMAX, NZ = 15, 6
PI = np.pi


@pytest.fixture(scope="module")
def plan():
    return O.Plan(LMAX, NZ, nlat=3 * (LMAX + 1) // 2, nphi=3 * (LMAX + 1))


def _case(P, ic):
    cth, sth, ph = P.angles()
    z = np.zeros_like(cth)
    fr, ft, fp = z.copy(), z.copy(), z.copy()
    aq, as_, at = (np.zeros(P.nlm, dtype=complex) for _ in range(3))
    lm = P.lm
    if ic == 1:
        fr = cth.copy(); aq[lm(1, 0)] = np.sqrt(4 * PI / 3)
    elif ic == 2:
        ft = -sth; as_[lm(1, 0)] = np.sqrt(4 * PI / 3)
    elif ic == 3:
        fp = sth.copy(); at[lm(1, 0)] = np.sqrt(4 * PI / 3)
    elif ic == 4:
        ft = cth * np.cos(ph); fp = -np.sin(ph); as_[lm(1, 1)] = np.sqrt(2 * PI / 3)
    elif ic == 5:
        ft = -np.sin(ph); fp = -cth * np.cos(ph); at[lm(1, 1)] = np.sqrt(2 * PI / 3)
    elif ic == 6:
        p0, p1 = np.ones_like(cth), cth.copy()
        for k in range(1, LMAX):
            p0, p1 = p1, ((2 * k + 1) * cth * p1 - k * p0) / (k + 1)
        fr = p1; aq[lm(LMAX, 0)] = np.sqrt(4 * PI / (2 * LMAX + 1))
    elif ic == 7:
        ft = -LMAX * sth ** (LMAX - 1) * np.sin(LMAX * ph)
        fp = -LMAX * sth ** (LMAX - 1) * cth * np.cos(LMAX * ph)
        c = np.sqrt((2 * LMAX + 1) / (4 * PI))
        for k in range(1, LMAX + 1):
            c *= np.sqrt((2 * k - 1.0) / (2 * k))
        at[lm(LMAX, LMAX)] = 1 / (2 * c)
    else:
        fr = cth.copy(); ft = cth * np.cos(ph) - np.sin(ph); fp = -np.sin(ph) - cth * np.cos(ph)
        aq[lm(1, 0)] = np.sqrt(4 * PI / 3)
        as_[lm(1, 1)] = np.sqrt(2 * PI / 3)
        at[lm(1, 1)] = np.sqrt(2 * PI / 3)
    return [np.asarray(x, dtype=float) for x in (fr, ft, fp)], (aq, as_, at)


@pytest.mark.parametrize("ic", range(1, 9))
def test_known_answer(plan, ic):
    f, a = _case(plan, ic)
    k = np.arange(1, NZ + 1)
    grids = [k[:, None, None] * x[None] for x in f]
    specs = [k[:, None] * x[None] for x in a]
    got = plan.qst_analysis(*grids)
    for g, s in zip(got, specs):
        assert np.abs(g - s).max() < 1e-12
    back = plan.qst_synthesis(*specs)
    for g, s in zip(back, grids):
        assert np.abs(g - s).max() < 2e-12


def test_random_round_trip(plan):
    # prueba_vec.f90:100-129: S = 2Q, T = -Q, S00 = T00 = 0
    rng = np.random.default_rng(7)
    aq = rng.random(plan.nlm) - 0.5 + 1j * (rng.random(plan.nlm) - 0.5)
    aq[: LMAX + 1] = aq[: LMAX + 1].real
    as_, at = 2 * aq, -aq
    as_[0] = 0
    at[0] = 0
    k = np.arange(1, NZ + 1)[:, None]
    specs = [k * x[None] for x in (aq, as_, at)]
    back = plan.qst_analysis(*plan.qst_synthesis(*specs))
    for g, s in zip(back, specs):
        assert np.abs(g - s).max() < 1e-12
