"""The run loop (sph_run) against the oracle: ten RK3 steps of the vector
NL step at lmax 15, nz 64, with the energy history written to balance.txt,
the grid files of box_init (src/pseudo/pseudospec_mod.f90:204-220), and the
per-degree spectra, whose sum is the grid energy (FP64, 1e-12).  The oracle
runs on the extended-precision boundary matrices (oracle/extended.py), as
the CUDA path builds them."""
import os

import numpy as np
import pytest

from oracle import extended as X
from oracle import oracle as O
from tests._helpers import check, random_spec, rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12
NU, DT = 1e-3, 1e-4


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _state():
    P = O.Plan(15, 64, nlat=24, nphi=48, C=25, d=5, rint=0.5, rext=1.5)
    # the boundary matrices in long double, as the CUDA path builds them
    P.bc_setup(("noslip", "noslip"), tables=X.bc_tables(P, ("noslip", "noslip")))
    rng = np.random.default_rng(10)
    Z = random_spec(P, rng, power=3.0)
    W = random_spec(P, rng, power=3.0)
    Z, phi, W = P.imposebc(Z, P.dlr(W))
    return P, Z, W, phi


def _gpu(P):
    from redondito_b200 import sphp as S
    G = S.Plan(15, 64, nlat=24, nphi=48, Cz=25, oz=5, rint=0.5, rext=1.5)
    S.setup_bc(G)
    return S, G


@pytest.mark.parametrize("filt", [False, True])
def test_run_loop_energy_history(tmp_path, filt):
    P, Z, W, phi = _state()
    S, G = _gpu(P)
    # oracle loop: the step reports the energy of the state it starts from
    z, w, f = Z.copy(), W.copy(), phi.copy()
    energies, spectra = [], []
    for n in range(10):
        if n % 5 == 0:
            spectra.append(P.energy_spectrum(z, w))
        z, w, f, e = P.rk3_step(z, w, f, NU, DT)
        if filt:
            z, f = P.fc_filter(z, "r"), P.fc_filter(f, "r")
            z, f, w = P.imposebc(z, f)
        energies.append(e)
    spectra.append(P.energy_spectrum(z, w))
    energies.append(P.nl_rhs(z, w, f, NU)[2])
    Zg, Wg, Fg = dev(Z), dev(W), dev(phi)
    e_final = S.run(G, Zg, Wg, Fg, NU, DT, 10, tstep=1, sstep=5, filter=filt, outdir=str(tmp_path))
    torch.cuda.synchronize()
    bal = np.loadtxt(tmp_path / "balance.txt")
    assert bal.shape == (11, 3)
    assert np.array_equal(bal[:, 0], np.arange(11)) and np.allclose(bal[:, 1], np.arange(11) * DT)
    for n in range(11):
        check(abs(bal[n, 2] - energies[n]) / energies[n], TOL, f"energy of state {n}")
    check(abs(e_final - energies[-1]) / energies[-1], TOL, "final energy")
    for name, a, b in (("Z", Zg, z), ("W", Wg, w), ("phi", Fg, f)):
        # ten steps, each within 1e-12, the filtered run's rounding compounding
        check(rel_l2(a.cpu().numpy(), b), 3e-12, f"final {name}")
    for i, ref in enumerate(spectra):
        sp = np.loadtxt(tmp_path / f"lspectrum.{i:04d}.txt")
        assert sp.shape == (16, 3) and np.array_equal(sp[:, 0], np.arange(16))
        check(np.abs(sp[:, 1:] - ref).max() / np.abs(ref).max(), TOL, f"spectrum {i}")
    # the spectra sum to the energy of the state they describe
    s0 = np.loadtxt(tmp_path / "lspectrum.0000.txt")[:, 1:].sum()
    check(abs(s0 - energies[0]) / energies[0], TOL, "spectrum sum vs energy")
    G.close()


def test_grid_files(tmp_path):
    P, Z, W, phi = _state()
    S, G = _gpu(P)
    S.write_grids(G, str(tmp_path))
    th = np.loadtxt(tmp_path / "theta.txt")
    ph = np.loadtxt(tmp_path / "phi.txt")
    zz = np.loadtxt(tmp_path / "z.txt")
    assert th.shape == (24,) and ph.shape == (48,) and zz.shape == (64 - 25,)
    check(np.abs(th - P.theta).max(), 1e-15)
    check(np.abs(ph - P.phi).max(), 1e-14)
    check(np.abs(zz - P.z[:39]).max(), 1e-15)
    # Fortran 1PE23.15: width 23, one digit before the point, 15 after
    line = open(tmp_path / "theta.txt").readline().rstrip("\n")
    assert len(line) == 23 and line.strip()[1] == "." and "E" in line
    G.close()


def test_energy_spectrum_against_oracle():
    P, Z, W, phi = _state()
    S, G = _gpu(P)
    sp = np.array(S.energy_spectrum(G, dev(Z), dev(W)))
    ref = P.energy_spectrum(Z, W)
    check(np.abs(sp - ref).max() / np.abs(ref).max(), TOL, "spectrum")
    e = S.nl_rhs(G, dev(Z), dev(W), dev(phi), NU, G.new_spec(), G.new_spec())
    check(abs(sp.sum() - e) / e, TOL, "Parseval")
    G.close()


def test_solver_command_line(tmp_path):
    """python -m redondito_b200.solver: namelist in, grid files, balance and
    spectra out, the final energy printed."""
    import json
    import subprocess
    import sys
    nml = tmp_path / "run.nml"
    nml.write_text("&grid lmax=15, nz=64, Cz=25, oz=5 /\n&boxparams rint=0.5d0, rext=1.5d0 /\n"
                   "&run dt=1d-4, step=4, tstep=2, sstep=2, nu=1d-3 /\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-m", "redondito_b200.solver", str(nml), str(tmp_path / "out"),
                          "--bc", "freeslip,noslip"], capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads(out.stdout.strip().splitlines()[-1])
    assert d["steps"] == 4 and d["energy"] > 0
    bal = np.loadtxt(tmp_path / "out" / "balance.txt")
    assert bal.shape == (3, 3) and np.array_equal(bal[:, 0], [0, 2, 4])
    assert abs(bal[-1, 2] - d["energy"]) <= 1e-15 * d["energy"] + 1e-300
    for i in range(3):
        assert (tmp_path / "out" / f"lspectrum.{i:04d}.txt").exists()
    for f in ("theta.txt", "phi.txt", "z.txt"):
        assert (tmp_path / "out" / f).exists()
