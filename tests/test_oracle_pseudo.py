"""Oracle operators vs prueba_pseudo.f90 (lmax=7, nz=128, r in [0.5,1.5]).

Field c_lm g(r) with g = e^r sin 3r (prueba_pseudo.f90:40-115).  The
reference publishes derivr' 2.3e-7, derivr'' 3.6e-5, D_l 2.8e-6 and a
filter change of 1.7e-11 (LEEME.md:45); laplang, multr, saxpby, copy and
prodvec are exact to round-off.
"""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def setup():
    P = O.Plan(7, 128, C=25, d=5, rint=0.5, rext=1.5)
    lmi = np.arange(1, P.nlm + 1)
    cl = (1.0 + 0.1 * lmi) + 1j * (0.5 - 0.05 * lmi)
    z = P.z

    def g(p):
        if p == 0:
            r = np.exp(z) * np.sin(3 * z)
        elif p == 1:
            r = np.exp(z) * (np.sin(3 * z) + 3 * np.cos(3 * z))
        else:
            r = np.exp(z) * (-8 * np.sin(3 * z) + 6 * np.cos(3 * z))
        return r[:, None] * cl[None]

    return P, g


def relerr(P, x, y):
    n = P.N
    return np.abs(x[:n] - y[:n]).max() / np.abs(y[:n]).max()


def within3(e, r):
    return r / 3 < e < 3 * r


def test_derivr(setup):
    P, g = setup
    a = g(0)
    b = P.derivr(a, 1)
    assert within3(relerr(P, b, g(1)), 2.3e-7)
    assert within3(relerr(P, P.derivr(a, 2), g(2)), 3.6e-5)
    c = P.derivr(P.z_forward(a), 1, "k")
    assert relerr(P, P.z_inverse(c), b) < 1e-14


def test_exact_ops(setup):
    P, g = setup
    a = g(0)
    ell = P.ell
    assert relerr(P, P.laplang(a), -(ell * (ell + 1))[None] * a) < 1e-15
    assert relerr(P, P.multr(a, -2), a / P.z[:, None] ** 2) < 1e-15
    b = P.derivr(a, 1)
    assert relerr(P, P.saxpby_c(a, 2.0, b, -3.0), 2 * a - 3 * b) < 1e-15
    assert relerr(P, P.copy(b), b) == 0.0


def test_dlr(setup):
    P, g = setup
    a = g(0)
    ex = g(2) - (P.ell * (P.ell + 1))[None] * a / P.z[:, None] ** 2
    assert within3(relerr(P, P.dlr(a), ex), 2.8e-6)


def test_fc_filter_change(setup):
    P, g = setup
    a = g(0)
    assert within3(relerr(P, P.fc_filter(a), a), 1.7e-11)
    # k-space form equals the r-space form
    k = P.fc_filter(P.z_forward(a), "k")
    assert relerr(P, P.z_inverse(k), P.fc_filter(a)) < 1e-15


def test_prodvec(setup):
    P, _ = setup
    th, ph, z = P.theta, P.phi, P.z
    T, F, Z = np.meshgrid(th, ph, z, indexing="ij")
    # grid layout (nz, nphi, nlat)
    T, F, Z = (x.transpose(2, 1, 0) for x in (T, F, Z))
    st, ct = np.sin(T), np.cos(T)
    u = (st * np.cos(F), Z, ct)
    v = (Z ** 2, np.sin(F), st * ct)
    w = P.prodvec(u, v)
    ex = (u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0])
    n = P.N
    for a, b in zip(w, ex):
        assert np.abs(a[:n] - b[:n]).max() < 1e-15
        assert np.all(a[n:] == 0.0)
