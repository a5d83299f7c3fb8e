"""The extended-precision boundary operators (oracle/extended.py) against
the oracle's restatement of invDl_setup / v_imposebc
(boundary_mod.f90:96-241, vboundary.f90:59-130).

Pins the long double evaluation by what holds for it exactly (B_l W = phi
on the interior rows, the wall rows of W), checks that the oracle's FFT-built
derivative matrices agree with it to their rounding, and measures the
oracle's own error on W and phi = D_l W: the error any FP64 restatement of
the reference's setup carries, and the reason the GPU's boundary outputs are
compared with the extended evaluation (tests/test_gpu_boundary_kinds.py,
tests/test_gpu_fullsize.py)."""
import numpy as np
import pytest

from oracle import extended as X
from oracle import oracle as O
from tests._helpers import check, random_spec

KINDS = [("noslip", "noslip"), ("freeslip", "freeslip"), ("freeslip", "noslip"), ("noslip", "freeslip")]


@pytest.fixture(scope="module")
def plan():
    return O.Plan(7, 64, C=25, d=5, rint=0.5, rext=1.5)


def test_derivative_matrices_match_the_oracle_to_its_rounding(plan):
    d1, d2 = X.derivr_matrices(plan)
    for order, de in ((1, d1), (2, d2)):
        do = plan.derivr_mat(order)
        err = float(np.abs(do - de.astype(np.float64)).max() / np.abs(de).max())
        check(err, 5e-13, f"derivr_mat order {order}, max entry error")


@pytest.mark.parametrize("kinds", KINDS)
def test_solve_is_exact_in_long_double(plan, kinds):
    rng = np.random.default_rng(4)
    phi = random_spec(plan, rng)
    W, F = X.imposebc_rows(plan, kinds, phi)
    n = plan.N
    sel = plan.ell > 0
    inner = F[2:n - 2, sel] - phi[2:n - 2, sel]
    # backward error of the long double solve: 1e-19 of |B| |W|, which is
    # about 1e3 |phi| here
    check(float(np.abs(inner).max() / np.abs(phi[2:n - 2]).max()), 1e-15, "D_l W - phi, interior")
    wmax = float(np.abs(W).max())
    assert np.abs(W[0]).max() <= 1e-16 * wmax and np.abs(W[n - 1]).max() <= 1e-16 * wmax
    d1, d2 = X.derivr_matrices(plan)
    z = plan.z
    for row, kind in ((0, kinds[0]), (n - 1, kinds[1])):
        cond = d1[row] @ W if kind == "noslip" else d2[row] @ W - 2 / X.L(z[row]) * (d1[row] @ W)
        check(float(np.abs(cond).max() / np.abs(d2[2:n - 2] @ W).max()), 1e-15, f"{kind} wall row {row}")


@pytest.mark.parametrize("kinds", KINDS)
def test_oracle_own_error(plan, kinds):
    """The reference's FP64 setup (restated by the oracle) against the
    extended evaluation: W within 1e-12, phi = D_l W within 3e-11 (no slip)
    and 3e-10 (a free-slip wall), printed."""
    plan.bc_setup(kinds)
    rng = np.random.default_rng(12)
    tor, phi = random_spec(plan, rng), random_spec(plan, rng)
    _, f_o, w_o = plan.imposebc(tor, phi)
    W, F = X.imposebc_rows(plan, kinds, phi)
    n = plan.N
    check(X.rel_l2(w_o[:n], W), 1e-12, f"oracle W {kinds}")
    check(X.rel_l2(f_o[:n], F), 3e-11 if kinds == ("noslip", "noslip") else 3e-10, f"oracle phi {kinds}")


@pytest.mark.parametrize("kinds", KINDS)
def test_oracle_with_extended_tables(plan, kinds):
    """The oracle's v_imposebc on the rounded extended tables: W to a few
    ulp; phi limited by the FP64 FFT second derivative (dlr)."""
    plan.bc_setup(kinds, tables=X.bc_tables(plan, kinds))
    rng = np.random.default_rng(12)
    tor, phi = random_spec(plan, rng), random_spec(plan, rng)
    _, f_o, w_o = plan.imposebc(tor, phi)
    W, F = X.imposebc_rows(plan, kinds, phi)
    n = plan.N
    check(X.rel_l2(w_o[:n], W), 1e-14, f"W {kinds}")
    check(X.rel_l2(f_o[:n], F), 3e-12, f"phi {kinds}")
    plan._bc = False  # the next test sets the oracle's own tables up again
