"""One field split over ranks (redondito_b200/slab.py), on CPU with gloo:
world sizes 2 and 3.  Each rank runs the 2D transforms of its planes and the
z transforms of its lm columns (here on the oracle, the checker of the
device path, so no GPU is needed) around the slab transposes; the split 3D
pair must equal the whole-field pair bit for bit, restricted to each
rank's part.  The transposes themselves are each other's inverse."""
import os
import socket

import numpy as np
import pytest

from redondito_b200 import slab

torch = pytest.importorskip("torch")
dist = pytest.importorskip("torch.distributed")

LMAX, NZ, NLAT, NPHI = 15, 64, 24, 48


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _whole(expect_dir):
    from oracle import oracle as O
    from tests._helpers import random_spec
    P = O.Plan(LMAX, NZ, nlat=NLAT, nphi=NPHI, C=25, d=5)
    rng = np.random.default_rng(4)
    grid = P.sh_synthesis(random_spec(P, rng))
    spec = P.forward_3d(grid)
    back = P.inverse_3d(spec)
    np.savez(os.path.join(expect_dir, "whole.npz"), grid=grid, spec=spec, back=back)


def _worker(rank, world, port, expect_dir):
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ref = np.load(os.path.join(expect_dir, "whole.npz"))
        k0, k1 = slab.bounds(NZ, world, rank)
        nlm = (LMAX + 1) * (LMAX + 2) // 2
        l0, l1 = slab.bounds(nlm, world, rank)
        Pa = O.Plan(LMAX, k1 - k0 + 1, nlat=NLAT, nphi=NPHI)  # the angular transforms of my planes
        Pz = O.Plan(LMAX, NZ, nlat=NLAT, nphi=NPHI, C=25, d=5)  # the z transforms
        # forward: 2D analysis of my planes, exchange, z forward of my columns
        carr = Pa.sh_analysis(ref["grid"][k0:k1 + 1])
        cols = slab.k_to_lm(torch.from_numpy(carr), NZ, nlm).numpy()
        spec = Pz.z_forward_cols(cols)
        assert np.array_equal(spec, ref["spec"][:, l0:l1 + 1])
        # inverse: z inverse of my columns, exchange, 2D synthesis of my planes
        zi = Pz.z_inverse_cols(spec)
        carr2 = slab.lm_to_k(torch.from_numpy(zi), NZ, nlm).numpy()
        back = Pa.sh_synthesis(carr2)
        assert np.array_equal(back, ref["back"][k0:k1 + 1])
        # the two transposes undo each other on arbitrary data
        rng = np.random.default_rng(rank)
        x = torch.from_numpy(rng.normal(size=(k1 - k0 + 1, nlm)) + 1j * rng.normal(size=(k1 - k0 + 1, nlm)))
        y = slab.lm_to_k(slab.k_to_lm(x, NZ, nlm), NZ, nlm)
        assert torch.equal(x, y)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_split_pair_equals_whole(tmp_path, world):
    _whole(str(tmp_path))
    torch.multiprocessing.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)


def test_bounds_match_range():
    """bounds is range (sphp_sca.F90:596-626) on [0, n): contiguous, in
    order, sizes differing by at most one, larger parts first."""
    for n in (1, 7, 64, 136, 131328):
        for world in range(1, 7):
            parts = [slab.bounds(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n - 1
            assert all(b[0] == a[1] + 1 for a, b in zip(parts, parts[1:]))
            sizes = [b - a + 1 for a, b in parts]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
