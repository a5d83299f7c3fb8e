"""Neumann and Robin reconstructions (fcgram_mod.f90:267-650), the wall
kinds of v_imposebc (vboundary.f90:59-130, noslip and freeslip) and the NL
step with free-slip walls on the GPU, against the oracle on the same inputs
and, for the boundary solve, against its extended-precision evaluation
(oracle/extended.py)."""
import numpy as np
import pytest

from oracle import extended as X
from oracle import oracle as O
from tests._helpers import check, random_spec, rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _pair(lmax=7, nz=128, nlat=None, nphi=None):
    from redondito_b200 import sphp as S
    P = O.Plan(lmax, nz, nlat=nlat, nphi=nphi, C=25, d=5, rint=0.5, rext=1.5)
    G = S.Plan(lmax, nz, nlat=P.nlat, nphi=P.nphi, Cz=25, oz=5, rint=0.5, rext=1.5)
    return S, P, G


@pytest.mark.parametrize("ord", [1, 2])
def test_neumann_reconstruct(ord):
    S, P, G = _pair()
    rng = np.random.default_rng(ord)
    f = random_spec(P, rng)
    for boun in (0, 1):
        ref = P.neumann_reconstruct(f, boun, ord)
        x = dev(f)
        S.neumann_reconstruct(G, x, boun, ord)
        check(rel_l2(x.cpu().numpy(), ref), 1e-15, f"neumann boun={boun} ord={ord}")
    G.close()


def test_robin_reconstruct():
    S, P, G = _pair()
    rng = np.random.default_rng(9)
    f = random_spec(P, rng)
    a = rng.normal(size=P.nlm)
    for boun in (0, 1):
        ref = P.robin_reconstruct(f, boun, a)
        x = dev(f)
        S.robin_reconstruct(G, x, boun, dev(a))
        check(rel_l2(x.cpu().numpy(), ref), 1e-15, f"robin boun={boun}")
    G.close()


KINDS = [("noslip", "noslip"), ("freeslip", "freeslip"), ("freeslip", "noslip"), ("noslip", "freeslip")]
TOL_W = 1e-14  # W = binv phi: binv correct to rounding, one FP64 product


@pytest.mark.parametrize("kinds", KINDS)
def test_imposebc_kinds(kinds):
    """v_imposebc and v_imposebc_fast for each pair of wall kinds:
    * against the oracle run on the extended-precision boundary tables (the
      same steps on the same matrices, to rounding): whole arrays, W within
      1e-12, phi within 1e-12 + 3x that oracle's own error for the field;
    * against the extended-precision values on the physical rows: W within
      1e-14, phi = D_l W (an FP64 FFT second derivative) within 1e-12 or 3x
      the oracle's own error on the same tables, whichever is larger;
    * against the oracle's own restatement of invDl_setup (FP64 matrices
      built by probing the FFT derivative): within that restatement's error
      against the extended values, printed."""
    S, P, G = _pair()
    Px = O.Plan(P.lmax, P.nz, C=25, d=5, rint=0.5, rext=1.5)
    P.bc_setup(kinds)
    Px.bc_setup(kinds, tables=X.bc_tables(Px, kinds))
    S.setup_bc(G, kinds)
    rng = np.random.default_rng(12)
    tor, phi = random_spec(P, rng), random_spec(P, rng)
    n = P.N
    w_x, f_x = X.imposebc_rows(P, kinds, phi)
    for fast in (False, True):
        t_ref, f_ref, w_ref = Px.imposebc(tor, phi, fast=fast)
        T, F, W = dev(tor), dev(phi), G.new_spec()
        (S.v_imposebc_fast if fast else S.v_imposebc)(G, T, F, W)
        t, f, w = T.cpu().numpy(), F.cpu().numpy(), W.cpu().numpy()
        check(rel_l2(t, t_ref), 1e-15, f"{kinds} tor fast={fast}")
        check(rel_l2(w, w_ref), TOL, f"{kinds} W vs oracle(extended tables) fast={fast}")
        check(X.rel_l2(w[:n], w_x), TOL_W, f"{kinds} W vs extended fast={fast}")
        # phi = D_l W by the FP64 FFT second derivative: its own rounding,
        # which the oracle on the same tables shows for this field
        e_x = X.rel_l2(f_ref[:n], f_x)
        print(f"oracle(extended tables) phi vs extended: {e_x:.2e}")
        check(rel_l2(f, f_ref), 3 * e_x + TOL, f"{kinds} phi vs oracle(extended tables) fast={fast}")
        check(X.rel_l2(f[:n], f_x), max(TOL, 3 * e_x), f"{kinds} phi vs extended fast={fast}")
        _, f_o, w_o = P.imposebc(tor, phi, fast=fast)
        ew, ef = X.rel_l2(w_o[:n], w_x), X.rel_l2(f_o[:n], f_x)
        print(f"reference setup (oracle, FP64 matrices) vs extended: W {ew:.2e} phi {ef:.2e}")
        check(rel_l2(w[:n], w_o[:n]), 2 * ew + TOL, f"{kinds} W vs oracle fast={fast}")
        check(rel_l2(f[:n], f_o[:n]), 2 * ef + TOL, f"{kinds} phi vs oracle fast={fast}")
    G.close()


def test_freeslip_needs_the_reconstructor():
    from redondito_b200 import sphp as S
    # a plan built with a continuation operator given directly has no Neumann tables
    dir_ = S.load_dirichlet_tables(25, 5)
    G = S.Plan(7, 64, Cz=25, oz=5, rint=0.5, rext=1.5, dir=dir_, tdir="/nonexistent")
    with pytest.raises(S.SphError) as e:
        S.setup_bc(G, ("freeslip", "noslip"))
    assert e.value.code == 4  # SPH_ENOTREADY
    S.setup_bc(G, ("noslip", "noslip"))
    G.close()


def test_freeslip_nl_step():
    """NL term and one RK3 step with free-slip walls, against the oracle on
    the extended-precision boundary tables."""
    S, P, G = _pair(lmax=15, nz=64, nlat=24, nphi=48)
    kinds = ("freeslip", "freeslip")
    P.bc_setup(kinds, tables=X.bc_tables(P, kinds))
    S.setup_bc(G, kinds)
    rng = np.random.default_rng(3)
    Z = random_spec(P, rng, power=3.0)
    W = random_spec(P, rng, power=3.0)
    Z, phi, W = P.imposebc(Z, P.dlr(W))
    rz_ref, rf_ref, e_ref = P.nl_rhs(Z, W, phi, 1e-3)
    rz, rf = G.new_spec(), G.new_spec()
    e = S.nl_rhs(G, dev(Z), dev(W), dev(phi), 1e-3, rz, rf)
    check(abs(e - e_ref) / e_ref, TOL, "energy")
    check(rel_l2(rz.cpu().numpy(), rz_ref), TOL, "rhs_z")
    check(rel_l2(rf.cpu().numpy(), rf_ref), TOL, "rhs_phi")
    Zr, Wr, Fr, e_ref = P.rk3_step(Z, W, phi, 1e-3, 1e-4)
    Zg, Wg, Fg = dev(Z), dev(W), dev(phi)
    S.rk3_step(G, Zg, Wg, Fg, 1e-3, 1e-4)
    for name, a, b in (("Z", Zg, Zr), ("W", Wg, Wr), ("phi", Fg, Fr)):
        check(rel_l2(a.cpu().numpy(), b), TOL, f"RK3 {name}")
    G.close()
