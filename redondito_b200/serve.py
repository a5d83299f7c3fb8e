"""Serving loop: continuous batching of transform and time-step requests,
admitted by HBM budget.

A request is a 3D transform pair of one scalar field (``"pair"``) or k RK3
steps of the vector nonlinear term with the Laplacian applied spectrally
(``"rk3"``), at one of several problem sizes.  Its work runs in a slot: a
plan with its scratch, a CUDA stream, and the request's spectral state.

Memory.  The first slot of a problem size creates a plan, with the
read-only device tables (Legendre tables, twiddles, tensor-core table tiles,
boundary matrices); every further slot of that size clones a plan of it
(sph_plan_clone), sharing those tables, with scratch of its own, so it costs
only its buffers and no host table work.  The tables go with the last slot
of the size.  A slot is kind-specific: a pair slot holds one spectrum and
one grid; an RK3 slot adds the nonlinear step's scratch (sph_setup_bc) and
the state (Z, W, phi).  The server keeps the bytes of its slots within
``hbm_budget``.

Admission.  Requests are admitted as they arrive.  A waiting request takes a
free slot of its (size, kind); without one, a new slot is created if it fits
the budget.  Otherwise a (size, kind) that already has a slot waits for it,
and one that has none releases idle slots of other (size, kind) until it
fits: clones first, least recently used first, the last slot of a size
(which holds its tables) only after them.  A request that still does not
fit waits until running slots finish.  The work of an
admitted request is queued at once on its slot's stream, so requests of all
sizes run side by side on the device; the host loop never blocks on the
device, it polls completion events.

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


def estimate_bytes(lmax, kind, precision_mixed):
    """Device bytes of a slot before it exists (a measured figure replaces
    it after the first one): the plan's scratch and the request state."""
    _, nz, nlat, nphi = size_of(lmax)
    nlm = (lmax + 1) * (lmax + 2) // 2
    ldn = (nlat // 2 + 3) // 4 * 4
    spec, grid = nz * nlm * 16, nz * nphi * nlat * 8
    g = 3 * (lmax + 1) * 2 * nz * ldn * 16
    b = g * (2 if precision_mixed else 1) + spec + grid
    if kind == "rk3":
        b += 15 * spec + 9 * grid
    return int(b * 1.05) + (1 << 20)


class Slot:
    """A plan of the slot's size (a clone of `source`, or a new plan with the
    tables when there is none), a stream, the state of its kind."""

    def __init__(self, S, torch, lmax, kind, precision, source=None):
        self.S, self.torch, self.lmax, self.kind = S, torch, lmax, kind
        # cudaMalloc returns once the memory is reserved, so the free-memory
        # delta needs no device synchronisation (which would stall the
        # requests running on the other slots' streams)
        free0 = torch.cuda.mem_get_info()[0]
        if source is not None:
            self.plan = source.clone()
        else:
            _, nz, nlat, nphi = size_of(lmax)
            self.plan = S.Plan(lmax, nz, nlat=nlat, nphi=nphi, Cz=25, oz=5, rint=0.5, rext=1.5, precision=precision)
        self.fresh = source is None
        P = self.plan
        if kind == "rk3":
            S.setup_bc(P)
        plan_bytes = max(0, free0 - torch.cuda.mem_get_info()[0])  # the plan's own cudaMalloc'd memory
        if kind == "rk3":
            self.Z, self.W, self.F = P.new_spec(), P.new_spec(), P.new_spec()
            state = (self.Z, self.W, self.F)
        else:
            self.a, self.grid = P.new_spec(), P.new_grid()
            state = (self.a, self.grid)
        self.stream = torch.cuda.Stream()
        self.event = torch.cuda.Event()
        self.bytes = plan_bytes + sum(x.numel() * x.element_size() for x in state)
        self.req = None
        self.last_used = 0.0

    def close(self):
        self.plan.close()
        for name in ("a", "grid", "Z", "W", "F"):
            if hasattr(self, name):
                delattr(self, name)


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


def pair_input(P, torch, rid):
    """The radial-space spectrum a pair request starts from."""
    return _seeded(P, torch, 1000 + rid, 2.0)


def launch(slot, req, nu=1e-3, dt=1e-5):
    """Queue the whole request on the slot's stream (no host synchronisation):
    a pair takes its seeded spectrum to (lm, kz), then runs the 3D inverse and
    forward transforms; an RK3 request imposes the no-slip rows on its seeded
    state and takes its steps."""
    S, torch, P, st = slot.S, slot.torch, slot.plan, slot.stream
    with torch.cuda.stream(st):
        if req.kind == "pair":
            slot.a.copy_(pair_input(P, torch, req.rid))
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
    """Slots created on demand within an HBM budget; continuous admission."""

    def __init__(self, S, torch, precision, hbm_budget, max_slots=None, clock=time.perf_counter):
        self.S, self.torch, self.precision = S, torch, precision
        self.budget = float(hbm_budget)
        self.max_slots = dict(max_slots or {})  # optional cap per (lmax, kind)
        self.slots = collections.defaultdict(list)
        self.measured = {}                       # (lmax, kind, fresh) -> bytes of such a slot
        self.bytes = 0
        self.peak_bytes = 0
        self.created = self.released = 0
        self.clock = clock

    # ------------------------------------------------------------ memory
    def _source(self, lmax):
        """A plan of this size to clone (any: they share the tables), or None."""
        for kind in ("pair", "rk3"):
            if self.slots[(lmax, kind)]:
                return self.slots[(lmax, kind)][0].plan
        return None

    def _need(self, lmax, kind, fresh):
        b = self.measured.get((lmax, kind, fresh))
        if b is None:
            b = self.measured.get((lmax, kind, True))
        if b is None:
            b = estimate_bytes(lmax, kind, self.precision == self.S.SPH_MIXED) * (2 if fresh else 1)
        return b

    def _release_idle(self, need, keep):
        """Release idle slots of other (size, kind) until `need` more bytes fit
        the budget; True if they do.  Slots whose size keeps another slot go
        first (least recently used first): releasing the last slot of a size
        frees its tables, and the next request of that size then builds them
        again on the host."""
        if self.bytes + need <= self.budget:
            return True
        count = collections.Counter(k[0] for k, ss in self.slots.items() for _ in ss)
        idle = sorted(((s.last_used, k, s) for k, ss in self.slots.items() if k != keep
                       for s in ss if s.req is None), key=lambda x: x[0])
        for keep_last in (True, False):  # first only slots that are not the last of their size
            for _, k, s in idle:
                if s not in self.slots[k] or (keep_last and count[k[0]] == 1):
                    continue
                count[k[0]] -= 1
                self.slots[k].remove(s)
                s.close()
                self.bytes -= s.bytes
                self.released += 1
                if self.bytes + need <= self.budget:
                    return True
        return False

    def _free_slot(self, lmax, kind, now):
        key = (lmax, kind)
        for s in self.slots[key]:
            if s.req is None:
                return s
        if self.max_slots.get(key) is not None and len(self.slots[key]) >= self.max_slots[key]:
            return None
        source = self._source(lmax)
        need = self._need(lmax, kind, source is None)
        if self.bytes + need > self.budget and self.slots[key]:
            # a (size, kind) that has a slot waits for it instead of pushing
            # other sizes out: every release frees device memory (a device-wide
            # synchronisation) and the next request of that size allocates again
            return None
        if not self._release_idle(need, key):
            return None
        if source is not None and self._source(lmax) is None:
            # releasing took the last plan of this size: the new slot builds the tables
            if not self._release_idle(self._need(lmax, kind, True), key):
                return None
        source = self._source(lmax)
        s = Slot(self.S, self.torch, lmax, kind, self.precision, source)
        self.measured[(lmax, kind, s.fresh)] = s.bytes
        self.bytes += s.bytes
        self.peak_bytes = max(self.peak_bytes, self.bytes)
        self.slots[key].append(s)
        self.created += 1
        return s

    def warm(self, keys):
        """Create one slot per (lmax, kind) ahead of the traffic, within the budget."""
        for lmax, kind in keys:
            s = self._free_slot(lmax, kind, 0.0)
            if s is not None:
                s.last_used = 0.0

    def reserve(self, counts):
        """Create slots ahead of the traffic: up to counts[(lmax, kind)] of
        each, in the order given, while they fit the budget without
        releasing any (later requests still create and release slots on
        demand).  Creating a slot allocates device memory, which a serving
        loop would otherwise do between requests."""
        for key, n in counts.items():
            need = lambda: self._need(key[0], key[1], self._source(key[0]) is None)
            while len(self.slots[key]) < n and self.bytes + need() <= self.budget:
                source = self._source(key[0])
                s = Slot(self.S, self.torch, key[0], key[1], self.precision, source)
                self.measured[(key[0], key[1], s.fresh)] = s.bytes
                self.bytes += s.bytes
                self.peak_bytes = max(self.peak_bytes, self.bytes)
                self.slots[key].append(s)
                self.created += 1

    def close(self):
        for ss in self.slots.values():
            for s in ss:
                s.close()
        self.slots.clear()
        self.bytes = 0

    # ------------------------------------------------------------ loop
    def serve(self, requests, keep_results=False):
        """Serve requests (arrival times in seconds from the start); returns
        them with t_admit / t_done filled in."""
        clock = self.clock
        waiting = collections.deque()
        running = []
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        t0 = clock()
        done = 0
        while done < len(requests):
            now = clock() - t0
            while pending and pending[0].arrival <= now:  # arrivals
                waiting.append(pending.popleft())
            still_waiting = collections.deque()
            while waiting:  # admission in arrival order; a request that cannot start waits
                r = waiting.popleft()
                s = self._free_slot(r.lmax, r.kind, now)
                if s is None:
                    still_waiting.append(r)
                    continue
                s.req, r.slot = r, s
                r.t_admit = clock() - t0
                s.last_used = r.t_admit
                launch(s, r)
                running.append(s)
            waiting = still_waiting
            if waiting and not running:
                # nothing runs and every idle slot of another size was released:
                # the first waiting request is larger than the budget
                raise MemoryError(f"request {waiting[0].rid} (lmax {waiting[0].lmax}, {waiting[0].kind}) "
                                  f"does not fit an HBM budget of {self.budget / 1e9:.1f} GB")
            still = []
            for s in running:  # completions
                if s.event.query():
                    r = s.req
                    r.t_done = clock() - t0
                    if keep_results:
                        r.result = [x.clone() for x in ((s.a,) if r.kind == "pair" else (s.Z, s.W, s.F))]
                    s.req = None
                    s.last_used = r.t_done
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
