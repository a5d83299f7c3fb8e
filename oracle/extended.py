"""Extended-precision (long double) evaluation of the boundary operators of
invDl_setup and v_imposebc (src/boundary/boundary_mod.f90:96-241,
src/boundary/vboundary.f90:59-130): the FC-Gram radial derivative matrices
on the N physical points, the matrices B_l and their inverse columns, and
W = B_l^-1 phi, phi' = D_l W on the physical rows.

TEST INFRASTRUCTURE, like the rest of oracle/: imported only by tests/.

Why.  The reference builds the derivative matrices in FP64 by probing its
FFT derivative with unit vectors (derivr_mat) and factors B_l in FP64.  The
entries carry rounding of about 1e-13 of the largest one, which B_l^-1 and
the second derivative of phi = D_l W amplify to 1e-11 (no slip) and 1e-10
(free slip) in phi.  The oracle restates that algorithm and so carries the
same error; the CUDA path builds the matrices in long double on the host.
Both approximate the values computed here: the same discrete operators (the
plan's continuation table dir and wavenumbers kz, as FP64 numbers) with
64-bit significands throughout, so that errors down to 1e-15 can be measured
and the oracle's own error stated.
"""
import numpy as np

L = np.longdouble
PI = L("3.14159265358979323846264338327950288")


def _derivr_operator(P, order):
    """(Dr, Di): long double nz x N, column j = the order-th FC-Gram radial
    derivative at the nz points (the N physical ones first) of the unit
    vector e_j (continued by
    the plan's table, transformed by a DFT over nz points, times (i kz)^order,
    transformed back), real and imaginary parts.  Di is not zero for odd
    orders when nz is even: the Nyquist wavenumber has one sign."""
    cache = P.__dict__.setdefault("_ext_dmat", {})
    if order in cache:
        return cache[order]
    n, nz = P.N, P.nz
    C = nz - n
    d = len(P.dir) // C
    dr = np.asarray(P.dir, dtype=L).reshape(d, C).T  # dir(ii, jj), column-major C x d
    f = np.zeros((nz, n), dtype=L)
    f[:n, :n] = np.eye(n, dtype=L)
    for ii in range(C):
        for jj in range(d):
            f[n + ii, n - d + jj] += dr[ii, jj]
            f[n + ii, d - 1 - jj] += dr[C - 1 - ii, jj]
    k = np.arange(nz)
    ang = -2 * PI * ((k[:, None] * k[None, :]) % nz).astype(L) / nz
    cs, sn = np.cos(ang), np.sin(ang)
    re, im = (cs @ f) / nz, (sn @ f) / nz
    kz = np.asarray(P.kz, dtype=L)[:, None]
    for _ in range(order):  # times i kz
        re, im = -kz * im, kz * re
    # inverse DFT (sign +1): cos(+a) = cs, sin(+a) = -sn; all nz rows
    cache[order] = (cs.T @ re + sn.T @ im, cs.T @ im - sn.T @ re)
    return cache[order]


def derivr_matrix(P, order):
    """derivr_mat (boundary_mod.f90:96-137) in long double: the real part of
    the order-th derivative of the unit vectors at the physical points, N x N."""
    return _derivr_operator(P, order)[0][:P.N]


def derivr_matrices(P):
    """(d1, d2) of derivr_matrix."""
    return derivr_matrix(P, 1), derivr_matrix(P, 2)


def derivr_rows(P, a, order):
    """derivr(a, order, 'r') of an FP64 spectral field a (nz, nlm): all nz
    rows (physical and continuation), complex long double (the operator is
    linear over the reals of each column: D a = (Dr + i Di) Re a + i (Dr +
    i Di) Im a)."""
    Dr, Di = _derivr_operator(P, order)
    x = np.asarray(a[:P.N])
    ar, ai = np.asarray(x.real, dtype=L), np.asarray(x.imag, dtype=L)
    return (Dr @ ar - Di @ ai) + 1j * (Di @ ar + Dr @ ai)


def _solve(B, rhs):
    """Gaussian elimination with partial pivoting, in long double."""
    B, rhs = B.copy(), rhs.copy()
    n = B.shape[0]
    for k in range(n):
        p = k + int(np.argmax(np.abs(B[k:, k])))
        if p != k:
            B[[k, p]] = B[[p, k]]
            rhs[[k, p]] = rhs[[p, k]]
        B[k + 1:, k] /= B[k, k]
        B[k + 1:, k + 1:] -= np.outer(B[k + 1:, k], B[k, k + 1:])
        rhs[k + 1:] -= np.outer(B[k + 1:, k], rhs[k])
    for k in range(n - 1, -1, -1):
        rhs[k] /= B[k, k]
        rhs[:k] -= np.outer(B[:k, k], rhs[k])
    return rhs


def _matrix(P, kinds, l):
    """B_l of invDl_setup for wall kinds (inner, outer): row 1 W = 0, row 2
    W' = 0 (noslip) or W'' - 2 W'/r = 0 (freeslip), rows 3..N-2 D_l, row N-1
    the outer wall's condition, row N W = 0."""
    d1, d2 = derivr_matrices(P)
    n = P.N
    z = np.asarray(P.z, dtype=L)
    B = np.zeros((n, n), dtype=L)
    B[0, 0] = 1
    B[1] = d2[0] - 2 / z[0] * d1[0] if kinds[0] == "freeslip" else d1[0]
    B[2:n - 2] = d2[2:n - 2]
    idx = np.arange(2, n - 2)
    B[idx, idx] -= L(l * (l + 1)) / z[idx] ** 2
    B[n - 2] = d2[n - 1] - 2 / z[n - 1] * d1[n - 1] if kinds[1] == "freeslip" else d1[n - 1]
    B[n - 1, n - 1] = 1
    return B


def binv(P, kinds, l):
    """M_l: columns 3..N-2 of B_l^-1 (N x (N-4), long double)."""
    n = P.N
    rhs = np.zeros((n, n - 4), dtype=L)
    rhs[np.arange(2, n - 2), np.arange(n - 4)] = 1
    return _solve(_matrix(P, kinds, l), rhs)


def bc_tables(P, kinds):
    """(binv, d2bor) rounded to FP64 in the oracle's layouts: binv (lmax, N-4,
    N) with [l-1, j, i] = M_l(i, j); d2bor (N, 4) with the rows 1, 2, N-1, N of
    d2 at [j, r]."""
    n = P.N
    out = np.zeros((max(P.lmax, 1), n - 4, n))
    for l in range(1, P.lmax + 1):
        out[l - 1] = binv(P, kinds, l).T.astype(np.float64)
    d2 = derivr_matrices(P)[1]
    d2bor = np.stack([d2[0], d2[1], d2[n - 2], d2[n - 1]], axis=1).astype(np.float64)
    return out, d2bor


def imposebc_rows(P, kinds, phi):
    """(W, D_l W) on the N physical rows, complex long double (N, nlm), for an
    FP64 spectral phi (nz, nlm): W = M_l phi(3..N-2) per column of degree l,
    zero for l = 0 (invDl), and its D_l = d2 - l(l+1)/r^2 (dlr)."""
    n = P.N
    d2 = derivr_matrices(P)[1]
    z = np.asarray(P.z, dtype=L)[:n, None]
    ell = np.asarray(P.ell)
    W = np.zeros((n, P.nlm), dtype=np.clongdouble)
    F = np.zeros((n, P.nlm), dtype=np.clongdouble)
    for l in range(1, P.lmax + 1):
        sel = ell == l
        w = binv(P, kinds, l) @ np.asarray(phi[2:n - 2, sel], dtype=np.clongdouble)
        W[:, sel] = w
        F[:, sel] = d2 @ w - (L(l * (l + 1)) / z ** 2) * w
    return W, F


def rel_l2(a, ref):
    """Relative L2 distance of an FP64 array from a long double one, taken in
    long double."""
    d = np.asarray(a, dtype=np.clongdouble) - ref
    return float(np.sqrt((np.abs(d) ** 2).sum() / (np.abs(ref) ** 2).sum()))
