"""Independent cross-checks of the oracle with third-party code present here:
scipy's Gauss-Legendre nodes and spherical harmonics, and numpy's FFT.  These
validate the oracle; they are never used as the oracle."""
import numpy as np
import pytest
import scipy.special as sp

from oracle import oracle as O


def test_gauss_nodes_weights():
    P = O.Plan(31, 4, nlat=48, nphi=96)
    x, w = sp.roots_legendre(48)
    assert np.abs(np.sort(P.ct) - np.sort(x)).max() < 1e-15
    assert np.abs(np.sort(P.w) - np.sort(w)).max() < 1e-14
    # exact for polynomials of degree < 2 nlat
    for k in range(0, 95, 7):
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs(np.sum(P.w * P.ct ** k) - exact) < 1e-15
    assert np.all(np.diff(P.ct) < 0)  # north pole first


def _Y(l, m, theta, phi):
    # scipy includes the Condon-Shortley phase; the reference's harmonics do not
    return (-1) ** m * sp.sph_harm_y(l, m, theta, phi)


def test_synthesis_matches_scipy_harmonics():
    lmax = 12
    P = O.Plan(lmax, 1, nlat=20, nphi=40)
    rng = np.random.default_rng(3)
    a = rng.normal(size=P.nlm) + 1j * rng.normal(size=P.nlm)
    a[P.emm == 0] = a[P.emm == 0].real
    g = P.sh_synthesis(a[None])[0]
    T, F = np.meshgrid(P.theta, P.phi)  # (nphi, nlat)
    ref = np.zeros_like(T)
    for idx in range(P.nlm):
        l, m = P.ell[idx], P.emm[idx]
        y = _Y(l, m, T, F)
        ref += (a[idx] * y).real if m == 0 else 2 * (a[idx] * y).real
    assert np.abs(g - ref).max() < 1e-12


def test_z_fft_matches_numpy():
    P = O.Plan(5, 58, nlat=8, nphi=16)
    rng = np.random.default_rng(5)
    f = rng.normal(size=(58, P.nlm)) + 1j * rng.normal(size=(58, P.nlm))
    assert np.abs(P.z_forward(f) - np.fft.fft(f, axis=0) / 58).max() < 1e-15
    assert np.abs(P.z_inverse(f) - np.fft.ifft(f, axis=0) * 58).max() < 1e-13


@pytest.mark.parametrize("nz", [33, 96, 11 * 13])
def test_generic_lengths(nz):
    P = O.Plan(3, nz, nlat=6, nphi=12)
    rng = np.random.default_rng(nz)
    f = rng.normal(size=(nz, P.nlm)) + 1j * rng.normal(size=(nz, P.nlm))
    assert np.abs(P.z_forward(f) - np.fft.fft(f, axis=0) / nz).max() < 1e-14
