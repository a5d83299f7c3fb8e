"""Multi-GPU sharding of independent units, on CPU with world_size 2 (gloo).

Every rank must compute the same greedy-by-flops assignment on its own
(no collective decides it), the shares must cover every unit exactly once,
and an ensemble run split across ranks must give, bit for bit, what one
process gives for every problem.  The work of each problem is the oracle's
(the checker of the device path), so this runs without a GPU."""
import os
import socket

import numpy as np
import pytest

from redondito_b200 import serve, shard

torch = pytest.importorskip("torch")
dist = pytest.importorskip("torch.distributed")

# (lmax, nz, nfields): a small ensemble of the benchmark ensemble's form
ENSEMBLE = [(15, 32, 1), (31, 32, 2), (15, 64, 3), (31, 64, 1), (15, 32, 2), (23, 32, 1), (31, 32, 3)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(lmax, nz, nf, seed):
    """The batch work of one problem on the oracle: per field a 3D inverse,
    a radial derivative and a 3D forward of the synthesised grid."""
    from oracle import oracle as O
    from tests._helpers import random_spec
    nlat = 3 * (lmax + 1) // 2
    P = O.Plan(lmax, nz, nlat=nlat, nphi=2 * nlat, C=25, d=5)
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nf):
        s = P.z_inverse(P.z_forward(random_spec(P, rng)))
        g = P.sh_synthesis(s)
        out.append((g, P.derivr(s, 1), P.forward_3d(g)))
    return out


def _worker(rank, world, port, expect_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard.ensemble_share(ENSEMBLE, rank, world)
        allp = [None] * world
        dist.all_gather_object(allp, (rank, mine, shard.ensemble_share(ENSEMBLE, 0, world)))
        # every rank derived the same assignment by itself
        assert all(p[2] == allp[0][2] for p in allp)
        got = {i: _problem(*ENSEMBLE[i], 100 + i) for i in mine}
        res = [None] * world
        dist.all_gather_object(res, got)
        if rank == 0:
            merged = {}
            for r in res:
                assert not set(r) & set(merged)
                merged.update(r)
            assert sorted(merged) == list(range(len(ENSEMBLE)))
            for i in range(len(ENSEMBLE)):
                ref = np.load(os.path.join(expect_dir, f"p{i}.npz"))
                for f, (g, d, o) in enumerate(merged[i]):
                    assert np.array_equal(g, ref[f"g{f}"]) and np.array_equal(d, ref[f"d{f}"])
                    assert np.array_equal(o, ref[f"o{f}"])
        # the request stream: each rank serves the requests assigned to it
        reqs = serve.poisson_mix(60, rate=500.0, seed=9)
        share = shard.stream_share(reqs, rank, world, serve.size_of)
        ids = [None] * world
        dist.all_gather_object(ids, [r.rid for r in share])
        flat = [i for x in ids for i in x]
        assert sorted(flat) == [r.rid for r in reqs] and len(set(flat)) == len(flat)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_equals_one_process(tmp_path):
    for i, p in enumerate(ENSEMBLE):
        arrs = {}
        for f, (g, d, o) in enumerate(_problem(*p, 100 + i)):
            arrs.update({f"g{f}": g, f"d{f}": d, f"o{f}": o})
        np.savez(tmp_path / f"p{i}.npz", **arrs)
    torch.multiprocessing.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)


def test_greedy_partition_balance_and_determinism():
    rng = np.random.default_rng(3)
    costs = list(rng.pareto(1.5, size=200) + 1.0)
    for world in (1, 2, 3, 4, 8):
        parts = shard.greedy_partition(costs, world)
        assert parts == shard.greedy_partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        ld = shard.loads(parts, costs)
        # longest-first greedy: max load <= 4/3 of the optimum, which is >= max(mean, largest unit)
        lower = max(sum(costs) / world, max(costs))
        assert max(ld) <= 4.0 / 3.0 * lower + 1e-9


def test_greedy_partition_edge_cases():
    assert shard.greedy_partition([], 3) == [[], [], []]
    assert shard.greedy_partition([5.0], 4) == [[0], [], [], []]
    assert shard.greedy_partition([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.greedy_partition([1.0], 0)
    # loads 3|0, 3|1, 3|2, 3|3 (tie: rank 0), then 8|3
    assert shard.assign_stream([3.0, 1.0, 1.0, 1.0, 5.0], 2) == [0, 1, 1, 1, 0]


def test_flop_model_orders_sizes():
    sz = lambda l: serve.size_of(l)
    f = [shard.request_flops(*sz(l), "pair") for l in (31, 63, 127, 255, 511)]
    assert all(b > 4 * a for a, b in zip(f, f[1:]))  # ~ lmax^3 growth
    assert shard.request_flops(*sz(63), "rk3", 2) == 2 * shard.request_flops(*sz(63), "rk3", 1)
    assert shard.problem_flops(127, 64, 192, 384, 3) == 3 * shard.problem_flops(127, 64, 192, 384, 1)
