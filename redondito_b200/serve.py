"""Serving loop: continuous batching of transform and time-step requests.

A request is a 3D transform pair of one scalar field (``"pair"``) or k RK3
steps of the vector nonlinear term with the Laplacian applied spectrally
(``"rk3"``), at one of several problem sizes.  The server owns slots --
a plan with its scratch, a CUDA stream, and the request's spectral state --
created up front within an HBM budget.  Requests are admitted as they
arrive, into any free slot of their size; the work of every admitted
request is queued at once on its slot's stream, so requests of all sizes
run side by side on the device, and a slot frees (and the next waiting
request of that size is admitted) when its completion event fires.  The
host loop never blocks on the device: it polls events.

Latency of a request = completion time (host clock at the poll that saw
its event complete) - arrival time.  State stays on the device; results
are read back only when asked for (tests).
"""
import collections
import time

import numpy as np


class Request:
    __slots__ = ("rid", "arrival", "lmax", "kind", "steps", "t_admit", "t_done", "result", "slot")

    def __init__(self, rid, arrival, lmax, kind, steps=0):
        self.rid, self.arrival, self.lmax, self.kind, self.steps = rid, arrival, lmax, kind, steps
        self.t_admit = self.t_done = None
        self.result = None
        self.slot = None


def size_of(lmax):
    """(lmax, nz, nlat, nphi) of a request size: nlat = 3(lmax+1)/2 rounded to
    a multiple of 4 (Gauss points), nphi = 2 nlat, nz = lmax/2 rounded to a
    multiple of 16, at least 64 so that the C = 25, d = 5 FC-Gram
    continuation has room."""
    nlat = 4 * ((3 * (lmax + 1) // 2 + 3) // 4)
    nz = max(64, 16 * round(lmax / 2 / 16))
    return lmax, nz, nlat, 2 * nlat


class Slot:
    def __init__(self, S, torch, lmax, precision):
        self.S, self.torch = S, torch
        lmax, nz, nlat, nphi = size_of(lmax)
        free0 = torch.cuda.mem_get_info()[0]
        self.plan = S.Plan(lmax, nz, nlat=nlat, nphi=nphi, Cz=25, oz=5, rint=0.5, rext=1.5, precision=precision)
        S.setup_bc(self.plan)
        self.stream = torch.cuda.Stream()
        P = self.plan
        self.a = P.new_spec()
        self.grid = P.new_grid()
        self.Z, self.W, self.F = P.new_spec(), P.new_spec(), P.new_spec()
        self.event = torch.cuda.Event()
        torch.cuda.synchronize()
        self.bytes = free0 - torch.cuda.mem_get_info()[0]
        self.req = None

    def close(self):
        self.plan.close()


def _seeded(P, torch, seed, power):
    """Seeded spectrum N(0,1)(l+1)^-power times a smooth radial profile."""
    gen = torch.Generator(device=P.device)
    gen.manual_seed(seed)
    ell = P.ell.to(P.device).double()
    emm = P.emm.to(P.device)
    re = torch.randn((P.nz, P.nlm), generator=gen, device=P.device, dtype=torch.float64)
    im = torch.randn((P.nz, P.nlm), generator=gen, device=P.device, dtype=torch.float64)
    x = torch.complex(re, im) * ((ell + 1.0) ** -power)
    x[:, emm == 0] = x[:, emm == 0].real.to(torch.complex128)
    z = P.z.to(P.device)
    prof = torch.cos(np.pi * (z - P.rint) / (P.rext - P.rint)) + 0.5
    return (x * prof[:, None]).contiguous()


def launch(slot, req, nu=1e-3, dt=1e-5):
    """Queue the whole request on the slot's stream (no host synchronisation)."""
    S, torch, P, st = slot.S, slot.torch, slot.plan, slot.stream
    with torch.cuda.stream(st):
        if req.kind == "pair":
            slot.a.copy_(_seeded(P, torch, 1000 + req.rid, 2.0))
            S.fftp1d_real_to_complex_z(P, slot.a, stream=st)
            S.fftp3d_complex_to_real(P, slot.a, slot.grid, stream=st)
            S.fftp3d_real_to_complex(P, slot.grid, slot.a, stream=st)
        else:
            slot.Z.copy_(_seeded(P, torch, 2000 + req.rid, 3.0))
            slot.W.copy_(_seeded(P, torch, 3000 + req.rid, 3.0))
            S.dlr(P, slot.W, slot.F, stream=st)
            S.v_imposebc(P, slot.Z, slot.F, slot.W, stream=st)
            for _ in range(req.steps):
                S.rk3_step(P, slot.Z, slot.W, slot.F, nu, dt, stream=st, energy=False)
        slot.event.record(st)


class Server:
    """Slots per request size within an HBM budget; continuous admission."""

    def __init__(self, S, torch, precision, slots_per_size, hbm_budget=None):
        self.S, self.torch = S, torch
        self.slots = collections.defaultdict(list)
        self.bytes = 0
        for lmax, n in slots_per_size.items():
            for _ in range(n):
                if hbm_budget is not None and self.slots[lmax] and self.bytes >= hbm_budget:
                    break  # budget reached: sizes keep at least one slot
                s = Slot(S, torch, lmax, precision)
                self.bytes += s.bytes
                self.slots[lmax].append(s)

    def close(self):
        for ss in self.slots.values():
            for s in ss:
                s.close()

    def serve(self, requests, keep_results=False, clock=time.perf_counter):
        """Serve requests (arrival times in seconds from the start, sorted);
        returns them with t_admit / t_done filled in."""
        waiting = collections.defaultdict(collections.deque)
        running = []
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        t0 = clock()
        done = 0
        while done < len(requests):
            now = clock() - t0
            while pending and pending[0].arrival <= now:  # arrivals
                r = pending.popleft()
                waiting[r.lmax].append(r)
            for lmax, q in waiting.items():  # admission into free slots
                for s in self.slots[lmax]:
                    if not q:
                        break
                    if s.req is None:
                        r = q.popleft()
                        s.req, r.slot = r, s
                        r.t_admit = clock() - t0
                        launch(s, r)
                        running.append(s)
            still = []
            for s in running:  # completions
                if s.event.query():
                    r = s.req
                    r.t_done = clock() - t0
                    if keep_results:
                        r.result = [x.clone() for x in ((s.a,) if r.kind == "pair" else (s.Z, s.W, s.F))]
                    s.req = None
                    done += 1
                else:
                    still.append(s)
            running = still
        self.torch.cuda.synchronize()
        return requests


def poisson_mix(n, rate, seed, sizes=(31, 63, 127, 255, 511), weights=(8, 4, 2, 1, 1)):
    """n requests with Poisson arrivals (mean `rate` per second): size by the
    weights, half transform pairs, half k ~ U[1, 10] RK3 steps."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    p = np.asarray(weights, float) / sum(weights)
    out = []
    for i in range(n):
        lmax = int(rng.choice(sizes, p=p))
        if rng.random() < 0.5:
            out.append(Request(i, float(t[i]), lmax, "pair"))
        else:
            out.append(Request(i, float(t[i]), lmax, "rk3", int(rng.integers(1, 11))))
    return out


def latency_stats(reqs):
    lat = np.array([r.t_done - r.arrival for r in reqs]) * 1e3
    span = max(r.t_done for r in reqs) - min(r.arrival for r in reqs)
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "jobs_per_s": len(reqs) / span, "jobs": len(reqs)}
