"""Shared helpers for the parity tests: seeded inputs and error measures."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)


def radial_profile(z, rint, rext, rng, kmax=8):
    """sum_k c_k cos(k pi (r - rint)/(rext - rint)), c_k ~ N(0,1)/(k+1)^2."""
    c = rng.normal(size=kmax + 1) / (np.arange(kmax + 1) + 1.0) ** 2
    return sum(c[k] * np.cos(k * np.pi * (z - rint) / (rext - rint)) for k in range(kmax + 1))


def random_spec(P, rng, power=2.0, radial=True):
    """a_lm(r) = N(0,1)(l+1)^-power (real for m = 0) times a smooth radial profile."""
    a = (rng.normal(size=P.nlm) + 1j * rng.normal(size=P.nlm)) * (P.ell + 1.0) ** -power
    a[P.emm == 0] = a[P.emm == 0].real
    if radial:
        prof = radial_profile(P.z, P.rint, P.rext, rng)
        return prof[:, None] * a[None, :]
    return np.repeat(a[None, :], P.nz, axis=0) * (1.0 + np.arange(P.nz))[:, None]


def check(err, tol, label=""):
    """Assert err < tol and print the measured figure (run pytest with -s to
    see every one): 'ERR <test>:<line> [label] <err> < <tol>'."""
    import inspect
    fr = inspect.stack()[1]
    print(f"ERR {fr.function}:{fr.lineno} {label} {err:.3e} < {tol:.0e}", flush=True)
    assert err < tol, f"{fr.function}:{fr.lineno} {label}: {err:.3e} >= {tol:.0e}"


def check_derivative(got, P, a, order, label="", floor=1e-12):
    """A CUDA radial derivative (derivr(a, order, 'r'), or dlr for order
    'dlr') of the FP64 spectral field a, as a numpy array, against the
    extended-precision operator (oracle/extended.py) and the oracle:

    * physical rows against the extended values: within max(floor, 3 x the
      oracle's own error there);
    * all nz rows (the continuation rows too) against the oracle: within
      3 x the oracle's own error on them + floor.

    A derivative of FP64 data carries rounding that the continuation and
    (i kz)^order amplify; the oracle's error shows how much for this field,
    so the bound follows the field instead of one number for every order."""
    from oracle import extended as X
    n = P.N
    if order == "dlr":
        x = X.derivr_rows(P, a, 2) - (P.ell * (P.ell + 1.0))[None, :] / np.asarray(P.z, dtype=X.L)[:, None] ** 2 \
            * np.asarray(a, dtype=np.clongdouble)
        o = P.dlr(a)
    else:
        x = X.derivr_rows(P, a, order)
        o = P.derivr(a, order)
    e_phys_o, e_all_o = X.rel_l2(o[:n], x[:n]), X.rel_l2(o, x)
    print(f"oracle {label} order {order}: physical rows {e_phys_o:.2e}, all rows {e_all_o:.2e} (vs extended)")
    check(X.rel_l2(got[:n], x[:n]), max(floor, 3 * e_phys_o), f"{label} order {order} physical rows vs extended")
    check(rel_l2(got, o), 3 * e_all_o + floor, f"{label} order {order} all rows vs oracle")
