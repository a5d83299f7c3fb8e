"""Tile-shape autotuner.

For a problem size (lmax, nz, nlat, nphi, precision) the tuner times the
candidate tile shapes of sph_plan_set_tiles -- MMA rows per scalar Legendre
work item (mixed plans), Gauss ring pairs per phi-transform CTA and lm
columns per z-transform CTA -- on the device and keeps the fastest.  A
timing is one batch run (3D pair plus radial derivative of one field, the
C4 work of a problem) of CONCURRENT copies of the problem, each on its own
plan, so that a shape is judged under the load of an ensemble rather than
alone (alone, shapes that split a small problem into more CTAs win, and
they lose when 64 problems share the device).  Results are cached in a JSON table keyed by the
problem size; the table measured on B200 ships as tiles_b200.json beside
this module and is what batches use by default.

    python -m redondito_b200.autotune --out redondito_b200/tiles_b200.json
"""
import argparse
import itertools
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tiles_b200.json")

ROWS = (64, 128)
RING_PAIRS = (2, 4, 8)
Z_COLS = (8, 16, 32, 64)
Z_SPLIT = (16, 32, 48, 64, 96, 128, 192, 256)  # z lengths whose width is fixed
CONCURRENT = 8  # problems per timed batch

# the C4 ensemble: lmax in {63, 127, 255}, nz in {32, 64, 96, 128}, nlat = 3(lmax+1)/2, nphi = 2 nlat
C4_LMAX = (63, 127, 255)
C4_NZ = (32, 64, 96, 128)


def key(lmax, nz, nlat, nphi, precision):
    return f"{'mixed' if precision else 'fp64'}/lmax{lmax}/nz{nz}/{nlat}x{nphi}"


def load_table(path=DEFAULT_TABLE):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_table(table, path):
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def candidates(lmax, nz, nlat, nphi, precision):
    """Tile shapes that sph_plan_set_tiles accepts for this size."""
    rows = ROWS if precision else (0,)
    # 0: the built-in choice (FP64: the cluster forward phi kernel where its
    # tiles divide nlat/2; mixed: the kernels chosen by the transform length)
    pairs = [0] + [r for r in RING_PAIRS if (nlat // 2) % r == 0 and r * nphi <= 8192]
    # the z lengths with a two-step kernel run at its compiled width
    cols = [0] if nz in Z_SPLIT else [c for c in Z_COLS if c * nz <= 4096]
    return [dict(rows=r, ring_pairs=p, z_cols=c) for r, p, c in itertools.product(rows, pairs, cols)]


def best(times):
    """The candidate with the smallest time: times is a list of (ms, tiles)."""
    return min(times, key=lambda t: t[0])[1] if times else None


def tiles_for(lmax, nz, nlat, nphi, precision, table=None):
    table = load_table() if table is None else table
    return table.get(key(lmax, nz, nlat, nphi, precision))


def apply(plan, tiles, S=None):
    if S is None:
        from redondito_b200 import sphp as S
    if tiles:
        S.set_tiles(plan, tiles["rows"], tiles["ring_pairs"], tiles["z_cols"])


def candidate_batch(S, plans, tiles):
    """The batch a candidate is timed on: the candidate's shape on every plan,
    and the shipped table NOT applied on top of it."""
    for P in plans:
        apply(P, tiles, S)
    return S.Batch(plans, [1] * len(plans), tuned=False)


def time_candidate(S, torch, plans, tiles, reps=5):
    """Device ms of one batch run (3D pair + radial derivative of one field
    per plan) with the candidate's tile shape."""
    B = candidate_batch(S, plans, tiles)
    P = plans[0]
    gen = torch.Generator(device=P.device)
    gen.manual_seed(1)
    for xs in B.spec:
        x = torch.randn((P.nz, P.nlm), generator=gen, device=P.device, dtype=torch.float64)
        xs[0].copy_(torch.complex(x, torch.zeros_like(x)))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    B.run()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        B.run()
    e1.record()
    torch.cuda.synchronize()
    B.status()
    B.close()
    return e0.elapsed_time(e1) / reps


def tune(lmax, nz, nlat, nphi, precision, reps=5, concurrent=CONCURRENT):
    import torch
    from redondito_b200 import sphp as S
    plans = [S.Plan(lmax, nz, nlat=nlat, nphi=nphi, Cz=25, oz=5,
                    precision=S.SPH_MIXED if precision else S.SPH_FP64) for _ in range(concurrent)]
    times = [(time_candidate(S, torch, plans, c, reps), c) for c in candidates(lmax, nz, nlat, nphi, precision)]
    for P in plans:
        P.close()
    t = best(times)
    return dict(t, ms=min(ms for ms, _ in times)), times


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    table = load_table(a.out)
    for precision, lmax, nz in itertools.product((0, 1), C4_LMAX, C4_NZ):
        nlat = 3 * (lmax + 1) // 2
        t, times = tune(lmax, nz, nlat, 2 * nlat, precision, a.reps)
        table[key(lmax, nz, nlat, 2 * nlat, precision)] = t
        print(key(lmax, nz, nlat, 2 * nlat, precision), t, flush=True)
    save_table(table, a.out)


if __name__ == "__main__":
    main()
