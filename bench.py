#!/usr/bin/env python
"""3D transform pairs/s at lmax=511, nr=256 on B200 (one line of JSON).

Workload (one "step" = one transform pair of the field set): a scalar field
and a vector field (3 components) at lmax = 511, Gauss grid 768 x 1536,
nz = 256 radial points with FC-Gram C = 25, d = 5 continuation, r in
[0.35, 1].  The state lives in (lm, kz) space; a pair is
    scalar: fftp3d_complex_to_real + fftp3d_real_to_complex
    vector: fftp3d_qst_to_vec + fftp3d_vec_to_qst (the z transforms of q,
            s, t composed with the 2D vector transforms)
Synthetic seeded inputs stand in for a simulation state: coefficients
N(0,1) (l+1)^-2.5 (real for m = 0) with 1% of the (r, l, m) entries set to
amplitude 1e3 and random phase, taken to (lm, kz) by the forward z
transform.  Every buffer is larger than L2 (126 MB), so no flush is needed.

  value   : pairs/s with the state resident in HBM (device events)
  e2e     : the same through the C ABI with host buffers: each step copies
            the 4 spectral fields host->device, runs the pair and copies
            them back (pinned memory, copies inside the timed region);
            neighbouring steps overlap on three state sets, uploads and
            downloads on their own streams
  roofline: the kernel class with the largest share of the timed region,
            achieved = algorithmic bytes (or flops) / its measured time
  cpu_baseline: the CPU oracle (a C++ restatement of the reference's
            arithmetic; the Fortran reference cannot be built here) timed
            on half of the pair (8 of its 16 slices, see CpuPair)
  fp64    : the FP64 form on the same state: pairs/s, per-kernel rooflines,
            e2e
  c1, c2  : configs 1 and 2 on the GPU and the CPU oracle (see config1,
            config2)

Multi-GPU: one process per GPU (torchrun); each rank runs its own replica
of the workload (a single problem does not shard: the reference's only
exchange is the slab transpose, which this design keeps on one device),
so scaling is weak and value is the sum over ranks of max-time throughput.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = dict(lmax=511, nlat=768, nphi=1536, nz=256, Cz=25, oz=5, rint=0.35, rext=1.0)
# a smaller case of the same kernels for ncu captures (each grid 150 MB, still > L2)
CASES = {"c3": W, "small": dict(lmax=255, nlat=384, nphi=768, nz=64, Cz=25, oz=5, rint=0.35, rext=1.0),
         # the benchmark's angular size on 32 planes (each grid 302 MB)
         "angular": dict(lmax=511, nlat=768, nphi=1536, nz=32, Cz=25, oz=5, rint=0.35, rext=1.0),
         # the benchmark's radial size on a quarter of its lm columns (each spectral field 135 MB)
         "radial": dict(lmax=255, nlat=384, nphi=768, nz=256, Cz=25, oz=5, rint=0.35, rext=1.0)}
METRIC = "3D transform pairs/s at lmax=511 nr=256"
SEED = 20261203 + 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="mixed (the headline, with the FP64 form timed beside it) or fp64")
    ap.add_argument("--no-fp64", action="store_true", help="mixed only: skip the FP64 comparison")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-f32", action="store_true", help="skip the single-precision-array pair")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the 64-problem batched ensemble")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--no-configs", action="store_true", help="skip the config 1 and config 2 blocks")
    ap.add_argument("--case", default="c3", choices=sorted(CASES),
                    help="c3: the benchmark workload; small, angular, radial: profiling cases for ncu")
    a = ap.parse_args()
    W.update(CASES[a.case]) if a.case != "c3" else None
    return a


# ---------------------------------------------------------------- CPU side
PAIR_SLICES = 16


class CpuPair:
    """The oracle's pair on the benchmark workload, cut into PAIR_SLICES equal
    slices.  Slice i runs, for all four fields, the z inverse of the lm
    columns [i nlm/S, (i+1) nlm/S), the angular synthesis (scalar and
    vector) and analysis of the planes [i nz/S, (i+1) nz/S), and the z
    forward (with the FC-Gram continuation) of the same columns.  The planes
    of the angular transforms are independent of one another and so are the
    columns of the z transforms, so S consecutive slices do exactly the
    arithmetic of one pair; nothing is extrapolated."""

    def __init__(self, threads=None):
        from oracle import oracle as O
        if threads:
            O.set_threads(threads)
        self.threads = O.lib().orc_get_threads()
        S = PAIR_SLICES
        lmax, nz = W["lmax"], W["nz"]
        assert nz % S == 0
        self.Pa = O.Plan(lmax, nz // S, nlat=W["nlat"], nphi=W["nphi"])
        self.Pz = O.Plan(lmax, nz, nlat=W["nlat"], nphi=W["nphi"], C=W["Cz"], d=W["oz"],
                         rint=W["rint"], rext=W["rext"])
        nlm = self.Pa.nlm
        self.cols = [(i * nlm) // S for i in range(S + 1)]
        rng = np.random.default_rng(SEED)
        amp = (self.Pa.ell + 1.0) ** -2.5
        self.spec = []
        for f in range(4):
            a = (rng.normal(size=(nz // S, nlm)) + 1j * rng.normal(size=(nz // S, nlm))) * amp
            a[:, self.Pa.emm == 0] = a[:, self.Pa.emm == 0].real
            if f >= 2:
                a[:, 0] = 0
            self.spec.append(a)
        self.zin = [rng.normal(size=(nz, nlm)) + 1j * rng.normal(size=(nz, nlm)) for _ in range(4)]

    def step(self, i):
        Pa, Pz = self.Pa, self.Pz
        c0, c1 = self.cols[i % PAIR_SLICES], self.cols[i % PAIR_SLICES + 1]
        zs = [Pz.z_inverse_cols(x[:, c0:c1]) for x in self.zin]
        g = Pa.sh_synthesis(self.spec[0])
        v = Pa.qst_synthesis(self.spec[1], self.spec[2], self.spec[3])
        Pa.sh_analysis(g)
        Pa.qst_analysis(*v)
        for x in zs:
            Pz.z_forward_cols(x)

    def sample(self):
        return (f"the oracle on all {self.threads} host threads, all 4 fields; a step is 1/{PAIR_SLICES} "
                f"of the pair: angular synthesis + analysis of {W['nz'] // PAIR_SLICES} of the {W['nz']} "
                f"planes and z inverse + forward of {self.cols[1]} of the {self.Pa.nlm} lm columns; "
                f"{PAIR_SLICES} consecutive steps cover one whole pair")


def cpu_pairs_per_s(nslices=PAIR_SLICES // 2, threads=None):
    """The oracle's pair throughput timed on `nslices` consecutive slices
    (half a pair by default, 10-20 s on the box's cores)."""
    cp = CpuPair(threads)
    cp.step(0)  # warm-up (page-in, thread pool)
    t0 = time.perf_counter()
    for i in range(nslices):
        cp.step(i)
    dt = time.perf_counter() - t0
    return (nslices / PAIR_SLICES) / dt, cp.threads, cp.sample() + f"; timed: {nslices} steps in {dt:.1f} s"


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cp = CpuPair()
    for i in range(args.warmup):
        cp.step(i)
    t0 = time.perf_counter()
    for i in range(args.steps):
        cp.step(i)
    dt = time.perf_counter() - t0
    v = (args.steps / PAIR_SLICES) / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "scalar + vector field, lmax=511, 768x1536, nz=256, FC-Gram C=25 d=5",
                   **W, "fields": 4, "step": f"1/{PAIR_SLICES} of the pair (see cpu_baseline.sample)"},
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cp.threads, "kind": "port",
                         "sample": cp.sample()},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (Fortran + SHTns + FFTW + MPI) cannot be built here; "
                "this is its C++ restatement (the oracle) on the host cores",
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- GPU side
def make_state(S, P, torch, gen):
    """4 spectral fields in (lm, kz): scalar a, vector q, s, t."""
    dev = P.device
    ell = P.ell.to(dev).double()
    emm = P.emm.to(dev)
    amp = (ell + 1.0) ** -2.5
    fields = []
    for f in range(4):
        re = torch.randn((P.nz, P.nlm), generator=gen, device=dev, dtype=torch.float64)
        im = torch.randn((P.nz, P.nlm), generator=gen, device=dev, dtype=torch.float64)
        x = torch.complex(re * amp, im * amp)
        spike = torch.rand((P.nz, P.nlm), generator=gen, device=dev) < 0.01
        ph = torch.rand((P.nz, P.nlm), generator=gen, device=dev, dtype=torch.float64) * 2 * np.pi
        x = torch.where(spike, 1e3 * torch.exp(1j * ph), x)
        x[:, emm == 0] = x[:, emm == 0].real.to(torch.complex128)
        if f >= 2:  # S and T have no l = 0 part
            x[:, 0] = 0
        x = x.contiguous()
        S.fftp1d_real_to_complex_z(P, x)
        fields.append(x)
    return fields


def pair(S, P, st, grids):
    a, q, s, t = st
    g0, g1, g2, g3 = grids
    S.fftp3d_complex_to_real(P, a, g0)
    S.fftp3d_qst_to_vec(P, q, s, t, g1, g2, g3)
    S.fftp3d_real_to_complex(P, g0, a)
    S.fftp3d_vec_to_qst(P, g1, g2, g3, q, s, t)


def pair32(S, P, st, grids):
    """The same pair with float grids and complex64 spectra (the
    single-precision entry points, a GSINGLE_PRECISION build's arrays)."""
    a, q, s, t = st
    g0, g1, g2, g3 = grids
    S.fftp3d_complex_to_real_f32(P, a, g0)
    S.fftp3d_qst_to_vec_f32(P, q, s, t, g1, g2, g3)
    S.fftp3d_real_to_complex_f32(P, g0, a)
    S.fftp3d_vec_to_qst_f32(P, g1, g2, g3, q, s, t)


def fp64_peak():
    from redondito_b200 import build as B
    try:
        out = subprocess.run([B.build_peak()], capture_output=True, text=True, timeout=120)
        return json.loads(out.stdout.strip().splitlines()[-1])["fp64_tensor_tflops"]
    except Exception:
        return None


# DRAM bytes per plane of one field of the two-pass forward phi transform
# (nphi 1536, lmax 511), from one ncu capture over 32 planes of the angular
# case: pass 1 read 307.4 MB and wrote 119.8 MB, pass 2 read 152.8 MB and
# wrote 105.8 MB.  The traffic grows in proportion to the planes, so a
# launch's traffic is this figure times the plane-fields it transforms.
PHI2_TRAFFIC_PER_PLANE = (307.4 + 119.8 + 152.8 + 105.8) / 32 * 1e6


def algorithmic_work(P, mixed):
    """Bytes (HBM kernels) or flops (Legendre) per step for each kernel class:
    compulsory reads + writes at their storage precision (grid FP64; folded
    coefficients FP64 complex, or in the mixed form bf16 x 3 pieces (12 B per
    complex) written by the forward phi FFT and fp32 complex read by the
    inverse; spectra FP64 complex); useful Legendre flops 4 nz (nlat/2) nlm
    per scalar direction (5x for a vector field)."""
    nlm, nz, nlat, nphi, lmax = P.nlm, P.nz, P.nlat, P.nphi, P.lmax
    grid_b = nlat * nphi * nz * 8
    cplx = (lmax + 1) * nlat * nz  # folded coefficients of one field (both parities)
    spec_b = nlm * nz * 16
    leg = 4.0 * nz * (nlat // 2) * nlm
    fwd_fold, inv_fold = (12, 8) if mixed else (16, 16)
    return {
        "phi_fwd": ("hbm", 4 * (grid_b + cplx * fwd_fold)),
        "phi_inv": ("hbm", 4 * (grid_b + cplx * inv_fold)),
        "zfft": ("hbm", 8 * 2 * spec_b),
        "leg_analysis": ("tensor", 2 * leg),
        "leg_synthesis": ("tensor", 2 * leg),
        "vec_analysis": ("tensor", 4 * leg),
        "vec_synthesis": ("tensor", 4 * leg),
        "ops": ("hbm", 0),
    }


def c4_ensemble(seed=20261203 + 4, nprob=64):
    """64 independent problems: lmax ~ U{63,127,255}, nz ~ U{32,64,96,128},
    nlat = 3(lmax+1)/2, nphi = 2 nlat, 1-3 fields, FC-Gram C=25 d=5, r in [0.35, 1]."""
    rng = np.random.default_rng(seed)
    return [(int(rng.choice((63, 127, 255))), int(rng.choice((32, 64, 96, 128))), int(rng.integers(1, 4)))
            for _ in range(nprob)]


def _max_over_ranks(torch, dist, world, x):
    if world > 1:
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        x = float(t.item())
    return x


def batched_c4(S, torch, steps, warmup, rank=0, world=1, dist=None):
    """The C4 ensemble as one batch per GPU (3D pair + radial derivative per
    field, one CUDA graph, grouped Legendre launches, autotuned tiles), FP64
    and mixed.  With several ranks each runs the problems the greedy-by-flops
    partition gives it; the run time is the max over ranks."""
    from redondito_b200 import shard
    ens = c4_ensemble()
    mine = shard.ensemble_share(ens, rank, world)
    nfield = sum(nf for _, _, nf in ens)
    out = {"problems": len(ens), "fields": nfield,
           "work": "per field: 3D inverse + radial derivative + 3D forward (one batch run)",
           "partition": "greedy by flops" if world > 1 else "one GPU"}
    for name, prec in (("fp64", S.SPH_FP64), ("mixed", S.SPH_MIXED)):
        plans = [S.Plan(ens[i][0], ens[i][1], nlat=3 * (ens[i][0] + 1) // 2, nphi=3 * (ens[i][0] + 1), Cz=25,
                        oz=5, rint=0.35, rext=1.0, precision=prec) for i in mine]
        B = S.Batch(plans, [ens[i][2] for i in mine]) if plans else None
        states = []
        for i, P, xs in zip(mine, plans, B.spec if B else []):
            gen = torch.Generator(device=P.device)
            gen.manual_seed(20261203 + 4 + 7919 * i)
            amp = (P.ell.to(P.device).double() + 1.0) ** -2.0
            for x in xs:
                re = torch.randn((P.nz, P.nlm), generator=gen, device=P.device, dtype=torch.float64)
                im = torch.randn((P.nz, P.nlm), generator=gen, device=P.device, dtype=torch.float64)
                v = torch.complex(re * amp, im * amp)
                v[:, P.emm.to(P.device) == 0] = v[:, P.emm.to(P.device) == 0].real.to(torch.complex128)
                x.copy_(v)
                S.fftp1d_real_to_complex_z(P, x)
                states.append(x.clone())
        for _ in range(warmup if B else 0):
            B.run()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps if B else 0):
            B.run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        rt = 0.0
        if B:
            B.status()
            rt = max(float((torch.linalg.vector_norm(x - r) / torch.linalg.vector_norm(r)).item())
                     for x, r in zip((x for xs in B.spec for x in xs), states))
            B.close()
        ms = _max_over_ranks(torch, dist, world, ms)
        rt = _max_over_ranks(torch, dist, world, rt)
        out[name] = {"ms_per_run": ms, "field_pairs_per_s": nfield / (ms * 1e-3),
                     "max_roundtrip_rel_l2": rt}
        for P in plans:
            P.close()
        del states
        torch.cuda.empty_cache()
    out["speedup_mixed_vs_fp64"] = out["fp64"]["ms_per_run"] / out["mixed"]["ms_per_run"]
    return out


def serving_c5(S, torch, nreq=200, rate=500.0, rank=0, world=1, dist=None, budget=120e9):
    """C5: Poisson arrivals (mean 500/s, seeded), sizes lmax 31/63/127/255/511
    weighted 8:4:2:1:1, half transform pairs, half k ~ U[1,10] RK3 steps;
    continuous admission into slots created on demand within an HBM budget
    (slots of one size share their tables).  Two runs per precision: the
    offered 500/s (above capacity: latency is queueing), and the same mix at
    half the measured capacity (latency is service).  With several ranks the
    stream is dispatched online to the least-loaded rank (by flops) and each
    rank runs its own server; latencies are pooled and the span is the
    longest over ranks."""
    from redondito_b200 import serve, shard
    sizes = (31, 63, 127, 255, 511)
    out = {"requests": nreq, "hbm_budget_gb": budget / 1e9,
           "sizes": {str(l): list(serve.size_of(l)[1:]) for l in sizes},
           "dispatch": "online least-loaded by flops" if world > 1 else "one GPU"}

    def run(srv, reqs):
        share = shard.stream_share(reqs, rank, world, serve.size_of)
        if world > 1:
            dist.barrier()
        srv.serve(share)
        lat = [(r.arrival, r.t_done) for r in share]
        if world > 1:
            allr = [None] * world
            dist.all_gather_object(allr, lat)
            lat = [x for r in allr for x in r]
        pooled = [serve.Request(i, a, 0, "pair") for i, (a, _) in enumerate(lat)]
        for r, (_, d) in zip(pooled, lat):
            r.t_done = d
        return serve.latency_stats(pooled)

    for name, prec in (("mixed", S.SPH_MIXED), ("fp64", S.SPH_FP64)):
        srv = serve.Server(S, torch, prec, hbm_budget=budget)
        warm = [serve.Request(i, 0.0, l, k, 1) for i, (l, k) in enumerate((l, k) for l in sizes
                                                                         for k in ("pair", "rk3"))]
        srv.serve(warm)
        # a slot pool sized for the mix (more slots for the frequent small
        # sizes), created before the traffic within the budget
        srv.reserve({(l, k): n for l, n in ((31, 4), (63, 4), (127, 2), (255, 2), (511, 1))
                     for k in ("pair", "rk3")})
        created0 = srv.created
        sat = run(srv, serve.poisson_mix(nreq, rate, seed=20261203 + 5))
        half = 0.5 * sat["jobs_per_s"]
        below = run(srv, serve.poisson_mix(nreq, half, seed=20261203 + 6))
        out[name] = {"offered_500_per_s": dict(sat, offered_per_s=rate),
                     "offered_half_capacity": dict(below, offered_per_s=half),
                     "slots_reserved": created0, "slots_created": srv.created - created0,
                     "slots_released": srv.released,
                     "peak_hbm_gb": srv.peak_bytes / 1e9}
        srv.close()
        torch.cuda.empty_cache()
    return out


def time_pairs(S, P, st, grids, steps, stream, torch, dist, world, fn=pair):
    """Device time of `steps` pairs (barrier + sync on both sides, max over ranks)."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn(S, P, st, grids)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=P.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def per_output_errors(S, Pm, Pd, st0, torch):
    """Each transform of the pair once on the same inputs in both forms: the
    inverse from the seeded spectra, the forward from the FP64 inverse's
    grids.  Relative L2 and max-abs (relative to max |FP64|) per output."""
    def inverse(P, spec):
        a, q, s, t = (x.clone() for x in spec)
        g = [P.new_grid() for _ in range(4)]
        S.fftp3d_complex_to_real(P, a, g[0])
        S.fftp3d_qst_to_vec(P, q, s, t, g[1], g[2], g[3])
        return g

    def forward(P, grids):
        out = [P.new_spec() for _ in range(4)]
        S.fftp3d_real_to_complex(P, grids[0], out[0])
        S.fftp3d_vec_to_qst(P, grids[1], grids[2], grids[3], out[1], out[2], out[3])
        return out

    rel, mx = {}, {}
    gd = inverse(Pd, st0)
    gm = inverse(Pm, st0)
    for name, a, b in zip(("grid_scalar", "grid_vr", "grid_vt", "grid_vp"), gm, gd):
        rel[name] = float((torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item())
        mx[name] = float(((a - b).abs().max() / b.abs().max()).item())
    del gm
    sd = forward(Pd, gd)
    sm = forward(Pm, gd)
    for name, a, b in zip(("spec_scalar", "Q", "S", "T"), sm, sd):
        rel[name] = float((torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item())
        mx[name] = float(((a - b).abs().max() / b.abs().max()).item())
    torch.cuda.synchronize()
    return rel, mx


def pair_parts(S, P, st, grids, f32=False):
    """The pair as four calls, each with the state fields it reads from the
    host upload and the fields whose final values it writes: (needs, call,
    finishes).  The scalar field (0) goes first in both directions, so its
    download overlaps the vector transforms."""
    sfx = "_f32" if f32 else ""
    a, q, s, t = st
    g0, g1, g2, g3 = grids
    fn = lambda name: getattr(S, name + sfx)
    return [((0,), lambda: fn("fftp3d_complex_to_real")(P, a, g0), ()),
            ((1, 2, 3), lambda: fn("fftp3d_qst_to_vec")(P, q, s, t, g1, g2, g3), ()),
            ((), lambda: fn("fftp3d_real_to_complex")(P, g0, a), (0,)),
            ((), lambda: fn("fftp3d_vec_to_qst")(P, g1, g2, g3, q, s, t), (1, 2, 3))]


E2E_MIN_STEPS = 12


def e2e_pairs(S, P, st, grids, steps, stream, torch, dist, world, f32=False):
    """The pair through the C ABI with host buffers: every step copies its four
    spectral fields from pinned host memory, runs the pair and copies the
    results back.  Steps are pipelined the way a streaming caller would run
    them: three device state sets, uploads on one stream, the pair on the
    compute stream, downloads on a third, so that the upload of step i+1 and
    the download of step i-1 overlap the pair of step i (the two copy
    directions use separate engines).  Within a step the copies go by field
    group: the scalar field's transforms start once it has landed, and its
    result goes back while the vector transforms run.  At least
    E2E_MIN_STEPS steps are timed, so that the pipeline's fill and drain
    (one upload and one download, about 40 ms each) do not dominate the
    figure; the steps run are in the result."""
    steps = max(steps, E2E_MIN_STEPS)
    NBUF = 3
    groups = [(0,), (1, 2, 3)]
    host_in = [x.cpu().pin_memory() for x in st]
    host_out = [[torch.empty_like(h).pin_memory() for h in host_in] for _ in range(NBUF)]
    bufs = [st] + [[x.clone() for x in st] for _ in range(NBUF - 1)]
    parts = [pair_parts(S, P, d, grids, f32) for d in bufs]
    nbytes = sum(h.numel() * h.element_size() for h in host_in)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev = lambda: torch.cuda.Event()
    in_done = [[ev() for _ in groups] for _ in range(NBUF)]
    fin = [[ev() for _ in groups] for _ in range(NBUF)]
    out_done = [ev() for _ in range(NBUF)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0.record(stream)
    s_in.wait_event(e0)
    s_out.wait_event(e0)
    for i in range(steps):
        b = i % NBUF
        d = bufs[b]
        if i >= NBUF:
            s_in.wait_event(out_done[b])  # this state set's previous results are on the host
        with torch.cuda.stream(s_in):
            for gi, grp in enumerate(groups):
                for f in grp:
                    d[f].copy_(host_in[f], non_blocking=True)
                in_done[b][gi].record(s_in)
        with torch.cuda.stream(stream):
            for needs, call, finishes in parts[b]:
                if needs:
                    stream.wait_event(in_done[b][groups.index(needs)])
                call()
                if finishes:
                    fin[b][groups.index(finishes)].record(stream)
        with torch.cuda.stream(s_out):
            for gi, grp in enumerate(groups):
                s_out.wait_event(fin[b][gi])
                for f in grp:
                    host_out[b][f].copy_(d[f], non_blocking=True)
        out_done[b].record(s_out)
    for b in range(min(NBUF, steps)):
        stream.wait_event(out_done[b])
    e1.record(stream)
    torch.cuda.synchronize()
    ems = _max_over_ranks(torch, dist, world, e0.elapsed_time(e1))
    del bufs, host_out, parts
    return {"value": world * steps / (ems * 1e-3), "unit": "pairs/s", "steps": steps,
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
            "pipeline": f"{NBUF} state sets; upload, pair and download of neighbouring steps overlap, "
                        "copies by field group (scalar, vector)"}


def kernel_rooflines(stage, work, steps, peaks, peak_fp64, fp64):
    """Per kernel class: algorithmic bytes (or useful flops) per step times the
    steps, over the class's event-timed duration; against the measured HBM
    copy bandwidth, or the tensor peak of the form (bf16 from the measured
    cuBLAS GEMM, FP64 from the DMMA probe run live)."""
    out = {}
    for c, (bound, per_step) in work.items():
        tms, nl = stage.get(c, (0.0, 0))
        if not nl or not per_step:
            continue
        if bound == "hbm":
            ach, peak, unit = per_step * steps / (tms * 1e-3) / 1e9, peaks.get("hbm_gbs", 6650.0), "GB/s"
        else:
            ach = per_step * steps / (tms * 1e-3) / 1e12
            peak, unit = (peak_fp64, "TFLOP/s") if fp64 else (peaks.get("bf16_tflops", 1590.0), "TFLOP/s")
        out[c] = {"bound": bound, "achieved": ach, "peak": peak, "unit": unit,
                  "frac": ach / peak if peak else None, "launches": nl, "ms_per_launch": tms / nl,
                  "ms_per_step": tms / steps}
    return out


def c1_seeded(P, rng):
    """Config 1 input: a_lm(r) = N(0,1)(l+1)^-2 (real for m = 0) times
    sum_k c_k cos(k pi (r - 0.35)/0.65), c_k ~ N(0,1)/(k+1)^2, k <= 8."""
    a = (rng.normal(size=P.nlm) + 1j * rng.normal(size=P.nlm)) * (P.ell + 1.0) ** -2.0
    a[P.emm == 0] = a[P.emm == 0].real
    c = rng.normal(size=9) / (np.arange(9) + 1.0) ** 2
    z = P.z
    prof = sum(c[k] * np.cos(k * np.pi * (z - 0.35) / 0.65) for k in range(9))
    return prof[:, None] * a[None, :]


def config1(S, torch, iters=200):
    """Config 1 (lmax 31, 48 x 96, r in [0.35, 1], C = 25, d = 5, nz = 33 and
    58): synthesis -> analysis -> derivr(., 1, 'r'), FP64, on the GPU (device
    time per chain over `iters` chains) and on the CPU oracle (all host
    threads), with the GPU outputs' relative L2 against the oracle's."""
    from oracle import oracle as O
    out = {}
    for nz in (33, 58):
        Po = O.Plan(31, nz, nlat=48, nphi=96, C=25, d=5, rint=0.35, rext=1.0)
        spec = c1_seeded(Po, np.random.default_rng(20261203 + 1))
        t0 = time.perf_counter()
        n_cpu = 0
        while n_cpu < 5 or time.perf_counter() - t0 < 1.0:
            g_ref = Po.sh_synthesis(spec)
            s_ref = Po.sh_analysis(g_ref)
            d_ref = Po.derivr(s_ref, 1)
            n_cpu += 1
        cpu_ms = 1e3 * (time.perf_counter() - t0) / n_cpu
        G = S.Plan(31, nz, nlat=48, nphi=96, Cz=25, oz=5, rint=0.35, rext=1.0)
        a = torch.from_numpy(spec).cuda()
        g, s, d = G.new_grid(), G.new_spec(), G.new_spec()

        def chain():
            S.fftp2d_complex_to_real_xy(G, a, g)
            S.fftp2d_real_to_complex_xy(G, g, s)
            S.derivr(G, s, d, 1, "r")
        for _ in range(20):
            chain()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(iters):
            chain()
        e1.record()
        torch.cuda.synchronize()
        gpu_ms = e0.elapsed_time(e1) / iters
        rel = lambda x, r: float(np.linalg.norm((x.cpu().numpy() - r).ravel()) / np.linalg.norm(r.ravel()))
        out[str(nz)] = {"gpu_ms_per_chain": gpu_ms, "cpu_ms_per_chain": cpu_ms, "cpu_over_gpu": cpu_ms / gpu_ms,
                        "rel_l2_vs_oracle": {"grid": rel(g, g_ref), "spec": rel(s, s_ref), "derivr": rel(d, d_ref)}}
        G.close()
    out["chain"] = "synthesis -> analysis -> derivr(.,1,'r'), FP64, one chain after another"
    return out


def config2(S, torch, cpu=True, reps=5):
    """Config 2 (lmax 255, 384 x 768, nz 128, C = 25, d = 5, r in [0.35, 1]):
    the vector nonlinear step from a no-slip state (Z, W ~ N(0,1)(l+1)^-3
    times a smooth radial profile, phi = D_l W, v_imposebc), FP64 and mixed
    on the GPU (device time per step over `reps` steps), the oracle on the
    host cores, and the GPU right-hand sides against the oracle's."""
    from oracle import oracle as O
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from tests._helpers import random_spec
    Po = O.Plan(255, 128, nlat=384, nphi=768, C=25, d=5, rint=0.35, rext=1.0)
    Po.bc_setup()
    rng = np.random.default_rng(20261203 + 2)
    Z0, W0 = random_spec(Po, rng, power=3.0), random_spec(Po, rng, power=3.0)
    Z, F, Wp = Po.imposebc(Z0, Po.dlr(W0))
    out = {"work": "one NL right-hand side (2 vector syntheses, 1 vector analysis, radial derivatives, "
                   "energy) from a no-slip state", "nu": 1e-3}
    ref = None
    if cpu:
        t0 = time.perf_counter()
        ref = Po.nl_rhs(Z, Wp, F, 1e-3)
        out["cpu_ms_per_step"] = 1e3 * (time.perf_counter() - t0)
        out["cpu_threads"] = O.lib().orc_get_threads()
    for name, prec in (("fp64", S.SPH_FP64), ("mixed", S.SPH_MIXED)):
        G = S.Plan(255, 128, nlat=384, nphi=768, Cz=25, oz=5, rint=0.35, rext=1.0, precision=prec)
        S.setup_bc(G)
        z, w, f = (torch.from_numpy(x).cuda() for x in (Z, Wp, F))
        rz, rf = G.new_spec(), G.new_spec()
        e = S.nl_rhs(G, z, w, f, 1e-3, rz, rf)
        S.nl_rhs(G, z, w, f, 1e-3, rz, rf)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            S.nl_rhs(G, z, w, f, 1e-3, rz, rf)
        e1.record()
        torch.cuda.synchronize()
        blk = {"gpu_ms_per_step": e0.elapsed_time(e1) / reps}
        if ref is not None:
            rel = lambda x, r: float(np.linalg.norm((x.cpu().numpy() - r).ravel()) / np.linalg.norm(r.ravel()))
            blk["rel_l2_vs_oracle"] = {"rhs_z": rel(rz, ref[0]), "rhs_phi": rel(rf, ref[1]),
                                       "energy": abs(e - ref[2]) / ref[2]}
            blk["cpu_over_gpu"] = out["cpu_ms_per_step"] / blk["gpu_ms_per_step"]
        out[name] = blk
        S.plan_status(G)
        G.close()
        torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import torch.distributed as dist
    from redondito_b200 import sphp as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))

    prec = S.SPH_FP64 if args.precision == "fp64" else S.SPH_MIXED
    mk = lambda pr: S.Plan(W["lmax"], W["nz"], nlat=W["nlat"], nphi=W["nphi"], Cz=W["Cz"], oz=W["oz"],
                           rint=W["rint"], rext=W["rext"], precision=pr)
    P = mk(prec)
    gen = torch.Generator(device=P.device)
    gen.manual_seed(SEED + rank)
    st = make_state(S, P, torch, gen)
    st0 = [x.clone() for x in st]
    grids = [P.new_grid() for _ in range(4)]
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        pair(S, P, st, grids)
    torch.cuda.synchronize()

    peak_fp64 = fp64_peak() if rank == 0 else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass

    gpu_index = local
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES")
    if cvd:
        try:
            gpu_index = int(cvd.split(",")[local])
        except ValueError:
            pass
    clk = ClockSampler(gpu_index)
    clk.start()
    time.sleep(0.3)

    S.timer_reset(P)
    S.timer_enable(P, True)
    ms = time_pairs(S, P, st, grids, args.steps, stream, torch, dist, world)
    S.timer_enable(P, False)
    clocks = clk.stop()
    stage = S.timer_read(P)
    ms_step = ms / args.steps
    value = world * args.steps / (ms * 1e-3)

    # a pair on a forward-transformed state is the identity up to rounding
    rt = [float((torch.linalg.vector_norm(x - r) / torch.linalg.vector_norm(r)).item()) for x, r in zip(st, st0)]

    e2e = None
    if not args.no_e2e:
        e2e = e2e_pairs(S, P, st, grids, args.steps, stream, torch, dist, world)

    # the same pair with the single-precision arrays on the mixed plan: device
    # time and e2e (float host buffers: half the bytes each way)
    single = None
    if prec == S.SPH_MIXED and not args.no_f32:
        st32 = [x.to(torch.complex64) for x in st0]
        g32 = [P.new_grid32() for _ in range(4)]
        for _ in range(max(1, args.warmup)):
            pair32(S, P, st32, g32)
        ms32 = time_pairs(S, P, st32, g32, args.steps, stream, torch, dist, world, fn=pair32)
        single = {"value": world * args.steps / (ms32 * 1e-3), "unit": "pairs/s", "ms_per_step": ms32 / args.steps,
                  "arrays": "float grids, complex64 spectra (sph_*_f32 on the mixed plan)"}
        if not args.no_e2e:
            single["e2e"] = e2e_pairs(S, P, st32, g32, args.steps, stream, torch, dist, world, f32=True)
        del st32, g32

    # the FP64 form on the same state: its time, per-kernel rooflines and e2e,
    # and the mixed form's error per output against it
    fp64 = None
    errors = None
    if prec == S.SPH_MIXED and not args.no_fp64:
        Pd = mk(S.SPH_FP64)
        std = [x.clone() for x in st0]
        gd = [Pd.new_grid() for _ in range(4)]
        for _ in range(max(1, args.warmup)):
            pair(S, Pd, std, gd)
        S.timer_reset(Pd)
        S.timer_enable(Pd, True)
        msd = time_pairs(S, Pd, std, gd, args.steps, stream, torch, dist, world)
        S.timer_enable(Pd, False)
        stage_d = S.timer_read(Pd)
        fp64 = {"value": world * args.steps / (msd * 1e-3), "unit": "pairs/s", "ms_per_step": msd / args.steps,
                "roofline": kernel_rooflines(stage_d, algorithmic_work(Pd, False), args.steps, peaks, peak_fp64,
                                             True),
                "stage_share": {c: round(stage_d[c][0] / max(msd, 1e-9), 4) for c in stage_d if stage_d[c][1]},
                "gpu_launches": sum(v[1] for v in stage_d.values())}
        if not args.no_e2e:
            fp64["e2e"] = e2e_pairs(S, Pd, std, gd, args.steps, stream, torch, dist, world)
        del std, gd
        rel, mx = per_output_errors(S, P, Pd, st0, torch)
        errors = {"rel_l2_vs_fp64": rel, "max_abs_vs_fp64": mx,
                  "note": "each transform on the same inputs in both forms; both forms are checked against "
                          "the CPU oracle at this size (tests/test_gpu_fullsize.py)"}
        Pd.close()

    # roofline of the dominant kernel class, and every class's
    work = algorithmic_work(P, prec == S.SPH_MIXED)
    per_class = kernel_rooflines(stage, work, args.steps, peaks, peak_fp64, args.precision == "fp64")
    dom = max(stage, key=lambda c: stage[c][0])
    bound, per_step = work[dom]
    tms, nl = stage[dom]
    if bound == "hbm":
        achieved = per_step * args.steps / (tms * 1e-3) / 1e9
        peak = peaks.get("hbm_gbs", 6650.0)
        unit = "GB/s"
    else:
        achieved = per_step * args.steps / (tms * 1e-3) / 1e12
        peak = peak_fp64 if (peak_fp64 and args.precision == "fp64") else peaks.get("bf16_tflops", 1590.0)
        unit = "TFLOP/s"
    roofline = {"kernel": dom, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                "frac": achieved / peak if peak else None,
                "traffic": (PHI2_TRAFFIC_PER_PLANE * 4 * W["nz"] * args.steps / max(nl, 1)
                            if dom == "phi_fwd" and prec == S.SPH_MIXED and W["nphi"] == 1536 and W["lmax"] == 511
                            else None),
                "traffic_unit": "bytes per launch (ncu capture at 32 planes, scaled by plane-fields)",
                "launches": nl, "ms_per_launch": tms / max(nl, 1),
                "peak_source": ("fp64 DMMA probe run live (redondito_b200/peak/fp64_peak.cu)"
                                if bound == "tensor" and args.precision == "fp64"
                                else "measured (MEASURED_PEAKS.json)"
                                if ("hbm_gbs" if bound == "hbm" else "bf16_tflops") in peaks
                                else "fallback: this pool's earlier measurement, 6.65 TB/s and 1.59 PFLOP/s "
                                     "(MEASURED_PEAKS.json absent)")}
    shares = {c: round(stage[c][0] / max(ms, 1e-9), 4) for c in stage if stage[c][1]}
    launches = sum(v[1] for v in stage.values())

    c4 = None
    if not args.no_c4 and args.case == "c3":
        del grids
        torch.cuda.empty_cache()
        c4 = batched_c4(S, torch, args.steps, args.warmup, rank, world, dist)

    c5 = None
    if not args.no_serve and args.case == "c3":
        P.close()
        torch.cuda.empty_cache()
        c5 = serving_c5(S, torch, rank=rank, world=world, dist=dist)

    c1 = c2 = None
    if world == 1 and args.case == "c3" and not args.no_configs:
        c1 = config1(S, torch)
        c2 = config2(S, torch, cpu=not args.no_cpu)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, sample = cpu_pairs_per_s()
        cpu = {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": sample}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "bf16x3/f32",
        "data": "synthetic",
        "config": {"workload": (f"scalar + vector field, lmax={W['lmax']}, {W['nlat']}x{W['nphi']}, "
                                f"nz={W['nz']}, FC-Gram C={W['Cz']} d={W['oz']}"),
                   **W, "fields": 4, "precision": args.precision,
                   "l2_flush": "inputs larger than L2 (every buffer > 126 MB)",
                   "parallelism": f"replicas x{world}"},
        "e2e": e2e,
        "gpu_launches": launches,
        "roofline": roofline,
        "kernels": per_class,
        "stage_share": shares,
        "fp64": fp64,
        "single": single,
        "speedup_vs_fp64": (value / fp64["value"]) if fp64 else None,
        "accuracy": errors,
        "c1": c1,
        "c2": c2,
        "batched_c4": c4,
        "serve_c5": c5,
        "serve_p99_ms": c5["mixed"]["offered_half_capacity"]["p99_ms"] if c5 else None,
        "serve_p99_ms_offered_500": c5["mixed"]["offered_500_per_s"]["p99_ms"] if c5 else None,
        "roundtrip_rel_l2": {"scalar": rt[0], "Q": rt[1], "S": rt[2], "T": rt[3]},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
