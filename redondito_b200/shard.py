"""Spreading independent problems and requests over GPUs (one process per GPU).

A single shell problem does not shard in this design: the reference's only
exchange inside a problem is the slab all-to-all of its MPI decomposition
(src/sphp/sphp_sca.F90:629-760), and one B200 holds every problem of the
benchmark sizes whole.  What does shard is a set of independent units --
the problems of an ensemble, the requests of a serving stream -- and those
need no collective on the data path: every rank computes the same
assignment from the same unit list, runs its share with its own grouped
launches or server, and only the timings (and, when asked, results) are
gathered afterwards.

Assignment is greedy by work (longest-processing-time first): units sorted
by decreasing flop estimate, each given to the rank with the least work so
far, ties to the lowest rank.  Its most loaded rank carries at most 4/3 of
the optimum (Graham's bound).  A request stream, whose later arrivals are
not known when earlier ones are dispatched, is assigned online in arrival
order to the least-loaded rank.

The flop model counts the Legendre contractions (4 flop per complex x real
multiply-add, even/odd folded: 4 nz (nlat/2) nlm per scalar direction) and
the phi and z FFTs (5 N log2 N per complex length-N transform, halved for
the real-to-complex phi transforms).
"""
import math

# scalar-direction equivalents of the work units
VEC_DIRECTIONS = 5  # a vector (Q, S, T) direction = 5 scalar Legendre contractions
NL_STAGE_DIRECTIONS = 3 * VEC_DIRECTIONS  # u and w synthesised, u x w analysed
RK3_STAGES = 3


def direction_flops(lmax, nz, nlat, nphi):
    """Flops of one scalar 3D transform in one direction; nz counts the
    radial points including the continuation points (the FFT length)."""
    nlm = (lmax + 1) * (lmax + 2) // 2
    leg = 4.0 * nz * (nlat // 2) * nlm
    phi = 2.5 * nphi * math.log2(nphi) * nlat * nz
    zfft = 5.0 * nz * math.log2(nz) * nlm
    return leg + phi + zfft


def problem_flops(lmax, nz, nlat, nphi, nfields=1):
    """A batch problem: per field a 3D inverse, a radial derivative and a 3D forward."""
    nlm = (lmax + 1) * (lmax + 2) // 2
    return nfields * (2.0 * direction_flops(lmax, nz, nlat, nphi) + 5.0 * nz * math.log2(nz) * nlm)


def request_flops(lmax, nz, nlat, nphi, kind, steps=0):
    """A serving request: a scalar transform pair, or `steps` RK3 steps of the
    vector nonlinear term (three stages of three vector directions each)."""
    d = direction_flops(lmax, nz, nlat, nphi)
    if kind == "pair":
        return 2.0 * d
    return steps * RK3_STAGES * NL_STAGE_DIRECTIONS * d


def greedy_partition(costs, world):
    """Unit indices per rank: longest first, each to the least-loaded rank.

    Deterministic (ties by index, then by rank), so every rank that calls it
    with the same costs gets the same answer without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def assign_stream(costs, world):
    """Rank of each unit of a stream, assigned in arrival order to the rank
    with the least work assigned so far (ties to the lowest rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    out = []
    for c in costs:
        r = min(range(world), key=lambda r: (load[r], r))
        out.append(r)
        load[r] += c
    return out


def loads(parts, costs):
    return [sum(costs[i] for i in p) for p in parts]


def ensemble_share(ensemble, rank, world, size=lambda l: (3 * (l + 1) // 2, 3 * (l + 1))):
    """This rank's problems of an ensemble [(lmax, nz, nfields), ...]: the
    indices, in ensemble order.  size(lmax) gives (nlat, nphi)."""
    costs = [problem_flops(l, nz, *size(l), nf) for l, nz, nf in ensemble]
    return greedy_partition(costs, world)[rank]


def stream_share(requests, rank, world, size_of):
    """This rank's requests of a stream (Request objects sorted by arrival).
    size_of(lmax) gives (lmax, nz, nlat, nphi)."""
    costs = [request_flops(*size_of(r.lmax), r.kind, r.steps) for r in requests]
    ranks = assign_stream(costs, world)
    return [r for r, k in zip(requests, ranks) if k == rank]
