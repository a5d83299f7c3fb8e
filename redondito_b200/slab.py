"""One problem split over several GPUs: the slab transposes between ranks.

The reference splits a field over MPI ranks by planes (ksta..kend, physical
side) and by lm columns (lmsta..lmend, spectral side), both from range
(src/sphp/sphp_sca.F90:596-626), and exchanges the blocks between the 2D
transforms and the z transforms (fftp3d_redist_k_to_lm / _lm_to_k,
sphp_sca.F90:629-760).  Here one process drives one GPU and the exchange is
one all-to-all over torch.distributed (NCCL between GPUs; the functions
only move tensors, so any backend works -- the tests run them with gloo on
the CPU):

    k_to_lm(carr)  : this rank's per-plane spectra (nplanes, nlm) of planes
                     ksta..kend -> its columns (nz, nlm_local) of lmsta..lmend
    lm_to_k(spec)  : the reverse

and the 3D transforms of a split field built from the slab-local calls of
the C ABI (sph_plan_set_slab):

    fftp3d_real_to_complex(plan, grid_planes, spec_cols)
    fftp3d_complex_to_real(plan, spec_cols, grid_planes)   (spec_cols destroyed)

A field this large lives split because one GPU's HBM cannot hold it
(lmax >= 1023); a single problem that fits one GPU runs unsplit.  FP64 plans
only: the mixed form continues the physical planes before the angular
analysis, which needs the boundary planes of other ranks.
"""
import torch
import torch.distributed as dist


def bounds(n, nprocs, rank):
    """range (src/sphp/sphp_sca.F90:596-626), 0-based and inclusive: the part
    of [0, n) rank `rank` owns; the first mod(n, nprocs) ranks take one
    element more."""
    w1, w2 = divmod(n, nprocs)
    a = rank * w1 + min(rank, w2)
    return a, a + w1 - 1 + (1 if w2 > rank else 0)


def _world(group):
    return dist.get_rank(group), dist.get_world_size(group)


def _exchange(send_chunks, recv_counts, like, group):
    """all-to-all of complex chunks (one per destination rank, in rank order);
    returns the received chunks in source-rank order."""
    send = torch.cat([c.reshape(-1) for c in send_chunks]) if send_chunks else like.new_empty(0)
    recv = like.new_empty(sum(recv_counts))
    sr, rr = torch.view_as_real(send), torch.view_as_real(recv)
    dist.all_to_all_single(rr.reshape(-1), sr.reshape(-1), [2 * c for c in recv_counts],
                           [2 * c.numel() for c in send_chunks], group=group)
    return list(torch.split(recv, recv_counts))


def k_to_lm(carr, nz, nlm, group=None):
    """fftp3d_redist_k_to_lm: (nplanes, nlm) of this rank's planes ->
    (nz, nlm_local) of this rank's lm columns."""
    rank, world = _world(group)
    planes = [bounds(nz, world, r) for r in range(world)]
    cols = [bounds(nlm, world, r) for r in range(world)]
    k0, k1 = planes[rank]
    l0, l1 = cols[rank]
    if carr.shape != (k1 - k0 + 1, nlm):
        raise ValueError(f"expected this rank's planes as ({k1 - k0 + 1}, {nlm}), got {tuple(carr.shape)}")
    send = [carr[:, c0:c1 + 1].contiguous() for c0, c1 in cols]
    nl = l1 - l0 + 1
    recv = _exchange(send, [(q1 - q0 + 1) * nl for q0, q1 in planes], carr, group)
    out = carr.new_empty((nz, nl))
    for (q0, q1), chunk in zip(planes, recv):
        out[q0:q1 + 1] = chunk.view(q1 - q0 + 1, nl)
    return out


def lm_to_k(spec, nz, nlm, group=None):
    """fftp3d_redist_lm_to_k: (nz, nlm_local) of this rank's lm columns ->
    (nplanes, nlm) of this rank's planes."""
    rank, world = _world(group)
    planes = [bounds(nz, world, r) for r in range(world)]
    cols = [bounds(nlm, world, r) for r in range(world)]
    k0, k1 = planes[rank]
    l0, l1 = cols[rank]
    if spec.shape != (nz, l1 - l0 + 1):
        raise ValueError(f"expected this rank's columns as ({nz}, {l1 - l0 + 1}), got {tuple(spec.shape)}")
    send = [spec[q0:q1 + 1].contiguous() for q0, q1 in planes]
    npl = k1 - k0 + 1
    recv = _exchange(send, [npl * (c1 - c0 + 1) for c0, c1 in cols], spec, group)
    out = spec.new_empty((npl, nlm))
    for (c0, c1), chunk in zip(cols, recv):
        out[:, c0:c1 + 1] = chunk.view(npl, c1 - c0 + 1)
    return out


def _set_rank_slab(S, plan, group):
    rank, world = _world(group)
    k0, k1 = bounds(plan.nz, world, rank)
    l0, l1 = bounds(plan.nlm, world, rank)
    S.set_slab(plan, k0, k1 - k0 + 1, l0, l1 - l0 + 1)


def fftp3d_real_to_complex(plan, grid_planes, spec_cols, group=None):
    """fftp3d_real_to_complex (sphp_sca.F90:237-270) of a split field: the 2D
    analysis of this rank's planes, the exchange, the z forward transform
    (FC-Gram continuation included) of this rank's columns."""
    from . import sphp as S
    if plan.precision != S.SPH_FP64:
        raise ValueError("split 3D transforms need an FP64 plan")
    _set_rank_slab(S, plan, group)
    carr = plan.new_plane_spec()
    S.fftp2d_real_to_complex_xy(plan, grid_planes, carr)
    spec_cols.copy_(k_to_lm(carr, plan.nz, plan.nlm, group))
    S.fftp1d_real_to_complex_z(plan, spec_cols)


def fftp3d_complex_to_real(plan, spec_cols, grid_planes, group=None):
    """fftp3d_complex_to_real (sphp_sca.F90:400-433) of a split field: the z
    inverse of this rank's columns (in place), the exchange, the 2D
    synthesis of this rank's planes."""
    from . import sphp as S
    if plan.precision != S.SPH_FP64:
        raise ValueError("split 3D transforms need an FP64 plan")
    _set_rank_slab(S, plan, group)
    S.fftp1d_complex_to_real_z(plan, spec_cols)
    carr = lm_to_k(spec_cols, plan.nz, plan.nlm, group)
    S.fftp2d_complex_to_real_xy(plan, carr, grid_planes)
