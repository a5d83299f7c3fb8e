"""Generate the FC-Gram Dirichlet continuation tables A{C}-{d}.dat and Q{d}.dat.

The reference reads these two tables from a SPECTER `tables` directory
(src/sphp/fcgram_mod.f90:186-263, `load_dirichlet_tables`) and forms the
continuation operator ``dir = A . Q^T``.  The tables themselves are not part
of the reference, so this script builds them with the published FC-Gram
method (Bruno & Lyon, J. Comput. Phys. 229 (2010); Lyon, SIAM J. Sci. Comput.
33(6) (2011); Fontana, Bruno, Mininni & Dmitruk, Comput. Phys. Commun. 2020):

* Q (d x d): the Gram basis, i.e. the d polynomials of degree < d that are
  orthonormal on the d matching points x = 0, 1, ..., d-1 (grid units).
  Q[i, j] = p_j(x_i), obtained from a QR factorisation of the Vandermonde
  matrix with a positive diagonal in R.
* A (C x d): each Gram polynomial p_j is continued by a trigonometric
  polynomial g_j of period P = 2 (2d + C - 1) with K harmonics.  g_j is the
  least-squares fit, over an oversampled grid, of p_j on the matching
  interval [0, d-1] and of zero on [d+C, 2d+C-1] (where the next period's
  left matching points sit).  The system is solved by a truncated SVD in
  60-digit arithmetic.  A[c, j] = g_j(d + c), c = 0..C-1, the C points that
  follow the matching interval.

* Q1n (d x d) and Q2n (d x d), the Neumann tables of `load_neumann_tables`
  (fcgram_mod.f90:267-365), which forms the boundary reconstructor
  ``neu = Q(d,:) . Qn^T``: the value at the boundary point (x = d-1, the
  last matching point) from the other d-1 values and the first (Q1n) or
  second (Q2n) derivative there.  With M the d x d matrix whose rows
  0..d-2 are the Gram basis at x = 0..d-2 and whose last row is the basis'
  derivative of that order at x = d-1, the Gram coefficients of the
  interpolant are M^-1 [f_0..f_{d-2}, g], so Qn = (M^-1)^T.  The
  reconstructor reproduces polynomials of degree < d exactly.  The file
  starts with the table's grid spacing dxp (1: grid units), as the
  reference reads it.

The tables are written like the reference reads them: raw stream,
Fortran column-major float64 (`READ(10) A` on A(C,d), fcgram_mod.f90:234-248).

With d = 5, C = 25, K = 16 the radial derivative of sin(2.3z+0.4)+z^2 on
[0,1] has relative errors 2.48e-6, 4.92e-8, 2.19e-9 at nz = 64, 128, 256;
the reference publishes 2.5e-6, 4.9e-8, 2.2e-9 for its own tables.

Usage: python gen_fcgram.py [--C 25] [--d 5] [--out DIR]
"""
import argparse
import os

import mpmath as mp
import numpy as np


def gram_basis(d):
    """Q (d x d, columns = Gram polynomials on 0..d-1) and R with V = Q R."""
    V = mp.matrix(d, d)
    for i in range(d):
        for j in range(d):
            V[i, j] = mp.mpf(i) ** j
    Q, R = mp.qr(V)
    for j in range(d):
        if R[j, j] < 0:
            for i in range(d):
                Q[i, j] = -Q[i, j]
            for k in range(d):
                R[j, k] = -R[j, k]
    return Q, R


def continuation_table(d, C, K=16, over=10, cut=mp.mpf("1e-40")):
    Q, R = gram_basis(d)
    coef_poly = mp.inverse(R)  # p_j(x) = sum_k coef_poly[k, j] x^k
    P = mp.mpf(2 * (2 * d + C - 1))
    xs = [mp.mpf(i) / over for i in range((d - 1) * over + 1)]
    zs = [mp.mpf(d + C) + mp.mpf(i) / over for i in range((d - 1) * over + 1)]
    pts = xs + zs
    ncol = 2 * K + 1

    def basis_row(x):
        row = [mp.mpf(1)]
        for k in range(1, K + 1):
            a = 2 * mp.pi * k * x / P
            row += [mp.cos(a), mp.sin(a)]
        return row

    M = mp.matrix(len(pts), ncol)
    for r, x in enumerate(pts):
        for c, v in enumerate(basis_row(x)):
            M[r, c] = v
    U, S, Vt = mp.svd_r(M)
    A = np.zeros((C, d))
    cont_rows = [basis_row(mp.mpf(d + c)) for c in range(C)]
    for j in range(d):
        rhs = [sum(coef_poly[k, j] * x ** k for k in range(d)) for x in xs]
        rhs += [mp.mpf(0)] * len(zs)
        coef = [mp.mpf(0)] * ncol
        for s in range(ncol):
            if S[s] < cut * S[0]:
                continue
            ub = mp.fsum(U[r, s] * rhs[r] for r in range(len(pts)))
            for c in range(ncol):
                coef[c] += Vt[s, c] * ub / S[s]
        for c in range(C):
            A[c, j] = float(mp.fsum(a * b for a, b in zip(coef, cont_rows[c])))
    # entries that are zero in exact arithmetic come out near 1e-70: snap them
    Qd = np.array([[float(Q[i, j]) if abs(Q[i, j]) > 1e-40 else 0.0
                    for j in range(d)] for i in range(d)])
    return A, Qd


def neumann_table(d, order):
    """Qn = (M^-1)^T for the reconstruction from a derivative of `order`."""
    Q, R = gram_basis(d)
    coef = mp.inverse(R)  # p_j(x) = sum_k coef[k, j] x^k
    x = mp.mpf(d - 1)
    M = mp.matrix(d, d)
    for i in range(d - 1):
        for j in range(d):
            M[i, j] = Q[i, j]
    for j in range(d):
        if order == 1:
            M[d - 1, j] = mp.fsum(coef[k, j] * k * x ** (k - 1) for k in range(1, d))
        else:
            M[d - 1, j] = mp.fsum(coef[k, j] * k * (k - 1) * x ** (k - 2) for k in range(2, d))
    Mi = mp.inverse(M)
    return np.array([[float(Mi[j, i]) for j in range(d)] for i in range(d)])


def write_tables(outdir, C=25, d=5):
    mp.mp.dps = 60
    A, Q = continuation_table(d, C)
    os.makedirs(outdir, exist_ok=True)
    # Fortran column-major raw stream
    A.T.astype("<f8").tofile(os.path.join(outdir, f"A{C}-{d}.dat"))
    Q.T.astype("<f8").tofile(os.path.join(outdir, f"Q{d}.dat"))
    for order in (1, 2):
        Qn = neumann_table(d, order)
        with open(os.path.join(outdir, f"Q{order}n{d}.dat"), "wb") as f:
            np.array([1.0], "<f8").tofile(f)  # dxp: the tables are in grid units
            Qn.T.astype("<f8").tofile(f)
    return A, Q


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--C", type=int, default=25)
    ap.add_argument("--d", type=int, default=5)
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    a = ap.parse_args()
    A, Q = write_tables(a.out, a.C, a.d)
    print(f"wrote A{a.C}-{a.d}.dat ({A.shape}), Q{a.d}.dat ({Q.shape}), Q1n{a.d}.dat and Q2n{a.d}.dat to {a.out}")
