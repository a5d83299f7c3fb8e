"""Serving loop, host side: request mixes, sizes and statistics."""
from redondito_b200 import serve


def test_poisson_mix_is_seeded_and_weighted():
    a = serve.poisson_mix(400, rate=500.0, seed=1)
    b = serve.poisson_mix(400, rate=500.0, seed=1)
    assert [(r.arrival, r.lmax, r.kind, r.steps) for r in a] == [(r.arrival, r.lmax, r.kind, r.steps) for r in b]
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    n31 = sum(r.lmax == 31 for r in a)
    n511 = sum(r.lmax == 511 for r in a)
    assert n31 > 4 * n511  # weights 8:1
    assert all(1 <= r.steps <= 10 for r in a if r.kind == "rk3")
    assert 0.35 < sum(r.kind == "pair" for r in a) / len(a) < 0.65
    span = a[-1].arrival
    assert 0.6 < len(a) / span / 500.0 < 1.4


def test_sizes_fit_the_plans():
    for lmax in (15, 31, 63, 127, 255, 511):
        l, nz, nlat, nphi = serve.size_of(lmax)
        assert nlat % 2 == 0 and nlat >= lmax + 1 and nphi > 2 * lmax
        assert nz % 16 == 0 and nz - 25 >= 5
    assert serve.size_of(511) == (511, 256, 768, 1536)


def test_latency_stats():
    rs = [serve.Request(i, 0.01 * i, 31, "pair") for i in range(100)]
    for i, r in enumerate(rs):
        r.t_admit = r.arrival
        r.t_done = r.arrival + 0.001 * (i + 1)
    st = serve.latency_stats(rs)
    assert abs(st["p50_ms"] - 50.5) < 0.6 and st["p99_ms"] > 98
    assert st["jobs"] == 100


def test_slot_estimates_grow_with_size_and_kind():
    sizes = (31, 63, 127, 255, 511)
    for mixed in (False, True):
        pairs = [serve.estimate_bytes(l, "pair", mixed) for l in sizes]
        rk3 = [serve.estimate_bytes(l, "rk3", mixed) for l in sizes]
        assert all(a < b for a, b in zip(pairs, pairs[1:]))
        assert all(p < r for p, r in zip(pairs, rk3))
    # an RK3 slot at lmax 511 holds the NL step's 9 grids and 15 spectra: tens of GB
    assert 25e9 < serve.estimate_bytes(511, "rk3", False) < 60e9


# ---------------------------------------------------------------- admission, on fake slots
import itertools
import types

import pytest


class _FakeEvent:
    def __init__(self):
        self.polls = 0

    def query(self):  # completes on the third poll after its launch
        self.polls -= 1
        return self.polls < 0


class _FakeSlot:
    live = 0

    def __init__(self, S, torch, lmax, kind, precision, source=None):
        self.lmax, self.kind, self.fresh = lmax, kind, source is None
        self.plan = ("plan", lmax)
        self.bytes = serve.estimate_bytes(lmax, kind, False) * (2 if self.fresh else 1)
        self.event = _FakeEvent()
        self.req, self.last_used = None, 0.0
        _FakeSlot.live += 1

    def close(self):
        _FakeSlot.live -= 1


def _fake_launch(slot, req):
    slot.event.polls = 2


@pytest.fixture
def fake_server(monkeypatch):
    monkeypatch.setattr(serve, "Slot", _FakeSlot)
    monkeypatch.setattr(serve, "launch", _fake_launch)
    S = types.SimpleNamespace(SPH_FP64=0, SPH_MIXED=1)
    torch = types.SimpleNamespace(cuda=types.SimpleNamespace(synchronize=lambda: None))
    _FakeSlot.live = 0

    def make(budget):
        tick = itertools.count()
        return serve.Server(S, torch, S.SPH_FP64, budget, clock=lambda: next(tick) * 1e-4)
    return make


def _fresh(lmax, kind="rk3"):
    return serve.estimate_bytes(lmax, kind, False) * 2


def test_admission_waits_for_a_running_slot_instead_of_failing(fake_server):
    """A request that does not fit while another runs waits; once that one
    completes, its idle slot is released and the waiting request starts."""
    srv = fake_server(_fresh(127) + 0.5 * _fresh(63))
    reqs = [serve.Request(0, 0.0, 127, "rk3", 1), serve.Request(1, 0.0, 63, "rk3", 1)]
    srv.serve(reqs)
    assert all(r.t_done is not None for r in reqs)
    assert reqs[1].t_admit >= reqs[0].t_done
    assert srv.released == 1 and srv.peak_bytes <= srv.budget


def test_admission_alternating_sizes_within_budget(fake_server):
    srv = fake_server(_fresh(127) + 0.5 * _fresh(63))
    reqs = [serve.Request(i, 2e-4 * i, (127, 63)[i % 2], "rk3", 1) for i in range(8)]
    srv.serve(reqs)
    assert all(r.t_done >= r.t_admit >= r.arrival for r in reqs)
    assert srv.released >= 3 and srv.peak_bytes <= srv.budget
    srv.close()
    assert _FakeSlot.live == 0


def test_admission_rejects_a_request_larger_than_the_budget(fake_server):
    srv = fake_server(0.5 * _fresh(127))
    with pytest.raises(MemoryError):
        srv.serve([serve.Request(0, 0.0, 127, "rk3", 1), serve.Request(1, 1.0, 63, "pair")])


def test_slots_of_one_size_are_reused_and_cloned(fake_server):
    srv = fake_server(10 * _fresh(63))
    reqs = [serve.Request(i, 0.0, 63, "pair") for i in range(3)]
    srv.serve(reqs)
    ss = srv.slots[(63, "pair")]
    assert len(ss) == 3 and [s.fresh for s in ss] == [True, False, False]
    more = [serve.Request(10 + i, 0.0, 63, "pair") for i in range(3)]
    srv.serve(more)
    assert srv.created == 3  # the idle slots took the second wave


def test_release_keeps_the_last_slot_of_a_size(fake_server):
    """Under budget pressure the clones of a size go before the last slot of
    another size (which holds the tables)."""
    srv = fake_server(10 * _fresh(63))
    srv.serve([serve.Request(i, 0.0, 63, "pair") for i in range(3)])
    srv.serve([serve.Request(10, 0.0, 31, "pair")])
    assert len(srv.slots[(63, "pair")]) == 3 and len(srv.slots[(31, "pair")]) == 1
    # room for a new slot as large as the 31 slot only if something goes: a 63
    # clone goes, not the 31 slot (the last of its size)
    clone = srv.slots[(63, "pair")][1].bytes
    srv.budget = srv.bytes + 0.5 * clone
    assert srv._release_idle(clone, keep=(127, "pair"))
    assert len(srv.slots[(31, "pair")]) == 1 and len(srv.slots[(63, "pair")]) == 2
    # when only last slots are left, they go too, least recently used first
    srv.budget = 0.5 * clone
    assert not srv._release_idle(clone, keep=(127, "pair"))
    assert sum(len(v) for v in srv.slots.values()) == 0


def test_reserve_fills_the_pool_within_the_budget(fake_server):
    srv = fake_server(3 * _fresh(63, "pair") + _fresh(31, "pair"))
    srv.reserve({(31, "pair"): 2, (63, "pair"): 9})
    assert len(srv.slots[(31, "pair")]) == 2
    assert 1 <= len(srv.slots[(63, "pair")]) < 9
    assert srv.bytes <= srv.budget and srv.released == 0
    fresh = [s.fresh for s in srv.slots[(63, "pair")]]
    assert fresh[0] and not any(fresh[1:])  # one plan with tables, the rest clones
