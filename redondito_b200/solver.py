"""Runs the time loop of the vector nonlinear step from a namelist file.

    python -m redondito_b200.solver run.nml OUTDIR [--precision fp64|mixed]
                                    [--bc noslip,noslip] [--seed N]

The namelist holds the reference's groups &grid (lmax, nz, Cz, oz) and
&boxparams (rint, rext) (src/pseudo/pseudospec_mod.f90:41-69,151-160) and
the loop's &run group (dt, step, tstep, sstep, nu, filter; see
sph_read_namelist).  The angular grid follows grid_init's rule: nlat the
smallest multiple of 4 not below 3(lmax+1)/2, nphi = 2 nlat.  The run
starts from a seeded state -- Z and W with coefficients N(0,1)(l+1)^-3
times a smooth radial profile, phi = D_l W, the walls' conditions imposed --
and writes theta.txt, phi.txt, z.txt, balance.txt and lspectrum.NNNN.txt to
OUTDIR (sph_run).  It prints one JSON line with the final energy.
"""
import argparse
import json
import os
import sys

import numpy as np
import torch

from . import sphp as S


def seeded_state(plan, seed):
    """Z, W ~ N(0,1)(l+1)^-3 (real for m = 0) times sum_k c_k cos(k pi x),
    c_k ~ N(0,1)/(k+1)^2, x = (r - rint)/(rext - rint); phi = D_l W."""
    rng = np.random.default_rng(seed)
    ell, emm = plan.ell.numpy(), plan.emm.numpy()
    x = ((plan.z - plan.rint) / (plan.rext - plan.rint)).numpy()
    out = []
    for _ in range(2):
        a = (rng.normal(size=plan.nlm) + 1j * rng.normal(size=plan.nlm)) * (ell + 1.0) ** -3.0
        a[emm == 0] = a[emm == 0].real
        c = rng.normal(size=9) / (np.arange(9) + 1.0) ** 2
        prof = sum(c[k] * np.cos(k * np.pi * x) for k in range(9))
        out.append(torch.from_numpy(np.ascontiguousarray(prof[:, None] * a[None, :])).to(plan.device))
    Z, W = out
    phi = plan.new_spec()
    S.dlr(plan, W, phi)
    return Z, W, phi


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("namelist")
    ap.add_argument("outdir")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--bc", default="noslip,noslip", help="inner,outer wall kinds: noslip or freeslip")
    ap.add_argument("--seed", type=int, default=20261203)
    a = ap.parse_args(argv)
    nl = S.read_namelist(a.namelist)
    nlat = S.nlat_for(nl["lmax"])
    plan = S.Plan(nl["lmax"], nl["nz"], nlat=nlat, nphi=2 * nlat, Cz=nl["Cz"], oz=nl["oz"], rint=nl["rint"],
                  rext=nl["rext"], precision=S.SPH_MIXED if a.precision == "mixed" else S.SPH_FP64)
    kinds = tuple(a.bc.split(","))
    S.setup_bc(plan, kinds)
    Z, W, phi = seeded_state(plan, a.seed)
    S.v_imposebc(plan, Z, phi, W)
    os.makedirs(a.outdir, exist_ok=True)
    e = S.run(plan, Z, W, phi, nl["nu"], nl["dt"], nl["step"], nl["tstep"], nl["sstep"], nl["filter"], a.outdir)
    if plan.precision == S.SPH_MIXED:
        S.plan_status(plan)
    print(json.dumps({"steps": nl["step"], "dt": nl["dt"], "energy": e, "outdir": a.outdir}), flush=True)
    plan.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
