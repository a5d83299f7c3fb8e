"""Oracle vs the known answers of the reference's prueba_sphp.f90 (2D scalar SHT).

Each case restates prueba_sphp.f90:121-184: a field on the lmax=15 Gauss grid
(nlat=24, nphi=48, nz=6 planes, plane k multiplied by k) and its exact
coefficients in orthonormal harmonics without the Condon-Shortley phase,
f = sum a_l0 Y_l0 + sum_{m>0} 2 Re(a_lm Y_lm).  The reference reports errors
of 1e-30 .. 1e-13 (LEEME.md:34); the bound here is 1e-12.
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
    a = np.zeros(P.nlm, dtype=complex)
    lm = P.lm
    if ic == 1:
        f = np.ones_like(cth); a[lm(0, 0)] = np.sqrt(4 * PI)
    elif ic == 2:
        f = cth.copy(); a[lm(1, 0)] = np.sqrt(4 * PI / 3)
    elif ic == 3:
        f = sth * np.cos(ph); a[lm(1, 1)] = np.sqrt(2 * PI / 3)
    elif ic == 4:
        f = sth * np.sin(ph); a[lm(1, 1)] = -1j * np.sqrt(2 * PI / 3)
    elif ic == 5:
        f = 3 * cth ** 2 - 1; a[lm(2, 0)] = 4 * np.sqrt(PI / 5)
    elif ic == 6:
        f = sth ** 2 * np.cos(2 * ph); a[lm(2, 2)] = 2 * np.sqrt(2 * PI / 15)
    elif ic == 7:
        p0, p1 = np.ones_like(cth), cth.copy()
        for k in range(1, LMAX):
            p0, p1 = p1, ((2 * k + 1) * cth * p1 - k * p0) / (k + 1)
        f = p1; a[lm(LMAX, 0)] = np.sqrt(4 * PI / (2 * LMAX + 1))
    elif ic == 8:
        f = sth ** LMAX * np.cos(LMAX * ph)
        c = np.sqrt((2 * LMAX + 1) / (4 * PI))
        for k in range(1, LMAX + 1):
            c *= np.sqrt((2 * k - 1.0) / (2 * k))
        a[lm(LMAX, LMAX)] = 1 / (2 * c)
    else:
        f = 2 - 3 * cth + sth * np.sin(ph) + 0.5 * sth ** 2 * np.cos(2 * ph)
        a[lm(0, 0)] = 2 * np.sqrt(4 * PI)
        a[lm(1, 0)] = -3 * np.sqrt(4 * PI / 3)
        a[lm(1, 1)] = -1j * np.sqrt(2 * PI / 3)
        a[lm(2, 2)] = np.sqrt(2 * PI / 15)
    return np.asarray(f, dtype=float), a


@pytest.mark.parametrize("ic", range(1, 10))
def test_known_answer(plan, ic):
    f, a = _case(plan, ic)
    k = np.arange(1, NZ + 1)
    grid = k[:, None, None] * f[None]
    spec = k[:, None] * a[None]
    got = plan.sh_analysis(grid)
    assert np.abs(got - spec).max() < 1e-12
    back = plan.sh_synthesis(spec)
    assert np.abs(back - grid).max() < 1e-12


def test_random_round_trip(plan):
    # prueba_sphp.f90:93-111: random coefficients, m = 0 real
    rng = np.random.default_rng(20261203)
    a = rng.random(plan.nlm) - 0.5 + 1j * (rng.random(plan.nlm) - 0.5)
    a[: LMAX + 1] = a[: LMAX + 1].real
    spec = np.arange(1, NZ + 1)[:, None] * a[None]
    back = plan.sh_analysis(plan.sh_synthesis(spec))
    assert np.abs(back - spec).max() < 1e-12


def test_lm_order_is_m_major(plan):
    # SHTns order, m = 0 first (prueba_sphp.f90:97 relies on it)
    assert plan.lm(0, 0) == 0 and plan.lm(LMAX, 0) == LMAX and plan.lm(1, 1) == LMAX + 1
    assert plan.lm(LMAX, LMAX) == plan.nlm - 1
    assert np.all(plan.emm[: LMAX + 1] == 0)
