"""Oracle Neumann and Robin reconstructions (fcgram_mod.f90:267-650) on the
radial boundaries of the (lm, z) layout, and the free-slip boundary kind.

The reconstructor of order `ord` recovers a boundary value from the ord-th
outward normal derivative there and the d-1 values inside; it is exact for
polynomials of degree < d (the Gram basis), and converges as dz^d for smooth
functions.  Robin: f' + a f = g.  Free slip (stress-free walls): W = 0,
W'' - 2 W'/r = 0, Z' - 2 Z/r = 0, the toroidal condition by the Robin
reconstruction (a = +2/rint inside, -2/rext outside)."""
import numpy as np
import pytest

from oracle import oracle as O


def _poly_field(P, rng, deg=4):
    """f(z) = sum_j c_j (z - rint)^j per lm column (complex c), with its first
    and second z-derivatives."""
    c = rng.normal(size=(deg + 1, P.nlm)) + 1j * rng.normal(size=(deg + 1, P.nlm))
    x = (P.z - P.rint)[:, None]
    f = sum(c[j][None] * x ** j for j in range(deg + 1))
    f1 = sum(j * c[j][None] * x ** (j - 1) for j in range(1, deg + 1))
    f2 = sum(j * (j - 1) * c[j][None] * x ** (j - 2) for j in range(2, deg + 1))
    return f, f1, f2


def test_tables_reproduce_polynomials():
    """neu from the generated tables: exact on degree < d in grid units."""
    d = 5
    for ord in (1, 2):
        neu = O.load_neumann(d, ord, 1.0)
        for deg in range(d):
            p = np.poly1d(np.random.default_rng(deg + 10 * ord).normal(size=deg + 1))
            pred = sum(neu[k] * p(k) for k in range(d - 1)) + neu[d - 1] * p.deriv(ord)(d - 1)
            assert abs(pred - p(d - 1)) < 1e-12 * max(1.0, abs(p(d - 1)))


@pytest.mark.parametrize("ord", [1, 2])
def test_neumann_exact_on_polynomials(ord):
    P = O.Plan(7, 128, C=25, d=5, rint=0.5, rext=1.5)
    rng = np.random.default_rng(ord)
    f, f1, f2 = _poly_field(P, rng)
    n = P.N
    for boun, row, sgn in ((0, 0, -1.0), (1, n - 1, 1.0)):
        g = f.copy()
        # outward normal derivative of order ord: -d/dz inside, +d/dz outside
        g[row] = sgn * f1[row] if ord == 1 else f2[row]
        out = P.neumann_reconstruct(g, boun, ord)
        err = np.abs(out[row] - f[row]).max() / np.abs(f[row]).max()
        assert err < 1e-11, (boun, ord, err)
        keep = np.ones(P.nz, bool)
        keep[row] = False
        assert np.array_equal(out[keep], g[keep])


def test_neumann_converges():
    """f = e^z sin(3z): the reconstruction error falls by about 2^d per grid
    doubling (order >= 4)."""
    errs = []
    for nz in (64, 128, 256):
        P = O.Plan(3, nz, C=25, d=5, rint=0.5, rext=1.5)
        z = P.z[:, None] * np.ones((1, P.nlm))
        f = np.exp(z) * np.sin(3 * z) + 0j
        f1 = np.exp(z) * (np.sin(3 * z) + 3 * np.cos(3 * z)) + 0j
        g = f.copy()
        g[P.N - 1] = f1[P.N - 1]
        out = P.neumann_reconstruct(g, 1, 1)
        errs.append(abs(out[P.N - 1, 0] - f[P.N - 1, 0]))
    orders = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(orders) > 4.0, (errs, orders)


def test_robin_exact_on_polynomials():
    P = O.Plan(7, 128, C=25, d=5, rint=0.5, rext=1.5)
    rng = np.random.default_rng(7)
    f, f1, _ = _poly_field(P, rng)
    a = rng.normal(size=P.nlm)
    n = P.N
    for boun, row, sgn in ((0, 0, -1.0), (1, n - 1, 1.0)):
        g = f.copy()
        g[row] = sgn * f1[row] + a * f[row]
        out = P.robin_reconstruct(g, boun, a)
        assert np.abs(out[row] - f[row]).max() / np.abs(f[row]).max() < 1e-11


@pytest.fixture(scope="module", params=[("freeslip", "freeslip"), ("freeslip", "noslip"), ("noslip", "freeslip")])
def freeslip(request):
    kinds = request.param
    P = O.Plan(7, 128, C=25, d=5, rint=0.5, rext=1.5)
    P.bc_setup(kinds)
    rng = np.random.default_rng(11)
    z = P.z[:, None]
    cl = rng.normal(size=P.nlm) + 1j * rng.normal(size=P.nlm)
    # Z = r^2 h(r) meets Z' - 2Z/r = 0 where h' = 0 and Z = 0 where h = 0:
    # h = cos(pi x/L) for free slip at both walls, cos(pi x/2L) for free slip
    # inside and no slip outside, sin(pi x/2L) the other way round (x = r - rint,
    # L = rext - rint); its wall values are then spoiled, for imposebc to restore
    x = (z - P.rint) / (P.rext - P.rint)
    h = {("freeslip", "freeslip"): np.cos(np.pi * x), ("freeslip", "noslip"): np.cos(0.5 * np.pi * x),
         ("noslip", "freeslip"): np.sin(0.5 * np.pi * x)}[kinds]
    zs = cl[None] * (z ** 2 * h)
    z0 = zs.copy()
    z0[0] += 0.3
    z0[P.N - 1] -= 0.2
    w0 = cl[None] * (np.exp(z) * np.cos(2 * z))
    tor, phi, pol = P.imposebc(z0, P.dlr(w0))
    return kinds, P, zs, tor, phi, pol


def test_freeslip_conditions(freeslip):
    kinds, P, zs, tor, phi, pol = freeslip
    n, ell = P.N, P.ell
    d1, d2 = P.derivr_mat(1), P.derivr_mat(2)
    neu = P.neu[0]
    for w, row in ((0, 0), (1, n - 1)):
        r = P.z[row]
        sel = ell > 0
        # W = 0 at every wall
        assert np.abs(pol[row, sel]).max() == 0.0
        if kinds[w] == "freeslip":
            # W'' - 2 W'/r = 0 (FC-Gram derivative matrices, as invDl_setup builds them)
            res = d2[row] @ pol[:n, sel] - 2.0 / r * (d1[row] @ pol[:n, sel])
            assert np.abs(res).max() / np.abs(d2[2:n - 2] @ pol[:n, sel]).max() < 1e-12
            # Z' - 2 Z/r = 0 through the Gram reconstructor: Z_wall = sum neu(k) Z(interior) / (a neu(d) + 1)
            a = 2.0 / r if w == 0 else -2.0 / r
            rows = [5 - k for k in range(1, 5)] if w == 0 else [n - 1 - 5 + k for k in range(1, 5)]
            rec = sum(neu[k - 1] * tor[rows[k - 1]] for k in range(1, 5)) / (a * neu[4] + 1.0)
            assert np.abs(rec - tor[row]).max() < 1e-14 * np.abs(tor).max()
            # the restored wall value is the smooth field's, to the reconstructor's
            # order (dz^5), and the FC-Gram radial derivative meets the condition
            assert np.abs(tor[row] - zs[row]).max() / np.abs(zs[:n]).max() < 1e-8
            dz = d1[row] @ tor[:n]
            assert np.abs(dz - 2.0 * tor[row] / r).max() / np.abs(tor[:n]).max() < 1e-5
        else:
            assert np.abs(d1[row] @ pol[:n, sel]).max() < 1e-12 * np.abs(pol[:n, sel]).max()
            assert np.abs(tor[row]).max() == 0.0


def test_freeslip_idempotent_and_dl(freeslip):
    kinds, P, zs, tor, phi, pol = freeslip
    tor2, phi2, pol2 = P.imposebc(tor, phi)
    assert np.abs(pol2 - pol).max() / np.abs(pol).max() < 1e-12
    assert np.abs(tor2 - tor).max() / np.abs(tor).max() < 1e-13
    n = P.N
    sel = P.ell > 0
    dl = P.dlr(pol)
    assert np.abs(dl[2:n - 2, sel] - phi[2:n - 2, sel]).max() / np.abs(phi[2:n - 2, sel]).max() < 1e-11
