"""Oracle no-slip boundary vs prueba_boundary.f90 (lmax=7, nz=128, r in [0.5,1.5]).

Published (LEEME.md:45): Z = 0 at the walls, dW/dr 1e-14, interior phi
3e-12, l = 0 zeroed, idempotence 2e-13, W vs W0 6e-8, fast vs full 3e-12.
"""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def state():
    P = O.Plan(7, 128, C=25, d=5, rint=0.5, rext=1.5)
    P.bc_setup()
    z, n = P.z, P.N
    r1, r2 = z[0], z[n - 1]
    lmi = np.arange(1, P.nlm + 1)
    cl = (1.0 + 0.1 * lmi) + 1j * (0.5 - 0.05 * lmi)
    z0 = cl[None] * (1 + np.exp(z) * np.sin(3 * z))[:, None]
    w0 = cl[None] * ((z - r1) ** 2 * (z - r2) ** 2 * np.exp(z))[:, None]
    f0 = P.dlr(w0)
    fi = f0.copy()
    fi[0] += 1.0
    fi[1] -= 2.0
    fi[n - 2] += 3.0
    fi[n - 1] -= 4.0
    fi[:, P.ell == 0] = 5 + 1j
    tor, phi, pol = P.imposebc(z0, fi)
    return P, z0, w0, f0, fi, tor, phi, pol


def test_walls_and_interior(state):
    P, z0, w0, f0, fi, tor, phi, pol = state
    n, ell = P.N, P.ell
    assert np.abs(tor[0]).max() == 0 and np.abs(tor[n - 1]).max() == 0
    assert np.abs(tor[1:n - 1] - z0[1:n - 1]).max() == 0 and np.abs(tor[n:] - z0[n:]).max() == 0
    d1 = P.derivr_mat(1)
    r1, r2 = P.z[0], P.z[n - 1]
    e3 = e4 = e6 = e8 = 0.0
    for lm in range(P.nlm):
        if ell[lm] == 0:
            assert np.abs(phi[:, lm]).max() == 0 and np.abs(pol[:, lm]).max() == 0
            continue
        wm = np.abs(pol[:n, lm]).max()
        e3 = max(e3, max(abs(pol[0, lm]), abs(pol[n - 1, lm])) / wm)
        e4 = max(e4, max(abs(d1[0] @ pol[:n, lm]), abs(d1[n - 1] @ pol[:n, lm])) * (r2 - r1) / wm)
        e6 = max(e6, np.abs(phi[2:n - 2, lm] - f0[2:n - 2, lm]).max() / np.abs(f0[2:n - 2, lm]).max())
        e8 = max(e8, np.abs(pol[:n, lm] - w0[:n, lm]).max() / np.abs(w0[:n, lm]).max())
    assert e3 == 0.0
    assert e4 < 1e-13
    assert e6 < 1e-11
    assert 6e-8 / 3 < e8 < 3 * 6e-8


def test_idempotent(state):
    P, z0, w0, f0, fi, tor, phi, pol = state
    _, _, pol2 = P.imposebc(tor, phi)
    assert np.abs(pol2 - pol).max() / np.abs(pol).max() < 1e-12


def test_fast_matches_full(state):
    P, z0, w0, f0, fi, tor, phi, pol = state
    tor3, phi3, pol3 = P.imposebc(z0, fi, fast=True)
    assert max(np.abs(pol3 - pol).max(), np.abs(tor3 - tor).max()) == 0.0
    n = P.N
    assert np.abs(phi3[:n] - phi[:n]).max() / np.abs(phi[:n]).max() < 1e-11


def test_w_solves_dl(state):
    # W from invDl satisfies D_l W = phi at rows 3..N-2 (boundary_mod.f90:244-252)
    P, z0, w0, f0, fi, tor, phi, pol = state
    n = P.N
    dl = P.dlr(pol)
    sel = P.ell > 0
    assert np.abs(dl[2:n - 2, sel] - fi[2:n - 2, sel]).max() / np.abs(fi[2:n - 2, sel]).max() < 1e-11
