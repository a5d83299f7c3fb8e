"""Tile-shape autotuner, host side: candidate sets, table keys and files."""
from redondito_b200 import autotune as A


def test_candidates_respect_the_entry_point_limits():
    for lmax, nz in ((63, 32), (255, 128)):
        nlat = 3 * (lmax + 1) // 2
        for prec in (0, 1):
            cs = A.candidates(lmax, nz, nlat, 2 * nlat, prec)
            assert cs
            assert any(c["ring_pairs"] == 0 for c in cs)  # the built-in choice is a candidate
            for c in cs:
                rp = c["ring_pairs"]
                assert rp == 0 or ((nlat // 2) % rp == 0 and rp * 2 * nlat <= 8192)
                assert c["z_cols"] * nz <= 4096
                assert (c["rows"] == 0) == (prec == 0)


def test_best_and_table_round_trip(tmp_path):
    times = [(3.0, {"rows": 64}), (1.5, {"rows": 128}), (2.0, {"rows": 32})]
    assert A.best(times) == {"rows": 128}
    assert A.best([]) is None
    path = str(tmp_path / "t.json")
    k = A.key(127, 64, 192, 384, 1)
    A.save_table({k: {"rows": 128, "ring_pairs": 8, "z_cols": 64, "ms": 1.0}}, path)
    table = A.load_table(path)
    assert A.tiles_for(127, 64, 192, 384, 1, table)["ring_pairs"] == 8
    assert A.tiles_for(127, 64, 192, 384, 0, table) is None
    assert A.load_table(str(tmp_path / "missing.json")) == {}


def test_shipped_table_covers_the_ensemble_if_present():
    table = A.load_table()
    if not table:
        return
    for prec in (0, 1):
        for lmax in A.C4_LMAX:
            for nz in A.C4_NZ:
                nlat = 3 * (lmax + 1) // 2
                t = A.tiles_for(lmax, nz, nlat, 2 * nlat, prec, table)
                assert t is not None
                shape = {k: t[k] for k in ("rows", "ring_pairs", "z_cols")}
                assert shape in A.candidates(lmax, nz, nlat, 2 * nlat, prec)


def test_candidates_are_timed_without_the_table():
    """Each plan of the timed batch gets the candidate's shape, and the batch
    is built with tuned=False, so the shipped table cannot replace it."""
    calls = []

    class FakeS:
        @staticmethod
        def set_tiles(plan, rows, ring_pairs, z_cols):
            calls.append((plan, rows, ring_pairs, z_cols))

        class Batch:
            def __init__(self, plans, nfields, tuned=True):
                self.plans, self.nfields, self.tuned = plans, nfields, tuned

    tiles = {"rows": 64, "ring_pairs": 4, "z_cols": 8}
    B = A.candidate_batch(FakeS, ["p0", "p1", "p2"], tiles)
    assert B.tuned is False and B.nfields == [1, 1, 1]
    assert calls == [(p, 64, 4, 8) for p in ("p0", "p1", "p2")]
