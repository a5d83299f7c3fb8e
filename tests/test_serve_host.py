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
