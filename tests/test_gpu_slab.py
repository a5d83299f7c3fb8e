"""Slab-local calls (sph_plan_set_slab), the way a multi-rank caller uses the
reference: every rank transforms its planes ksta..kend in 2D (the
per-rank carr1 of src/sphp-gpu/sphp_sca.F90:771-853), the ranks exchange
their blocks (fftp3d_redist_k_to_lm, emulated here by slicing one device
array), and every rank runs the z transforms and the operators on its lm
columns lmsta..lmend.  The ranks run one after another on one GPU with one
plan, their bounds from range (src/sphp/sphp_sca.F90:596-626).  A slab's
result must equal the whole-field result restricted to it, bit for bit:
every kernel computes each plane and each lm column independently."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from tests._helpers import random_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NPROCS = 3


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _ranges(S, n, nprocs):
    return [S.range_(0, n - 1, nprocs, r) for r in range(nprocs)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_slab_pipeline_equals_whole_field(precision):
    from redondito_b200 import sphp as S
    prec = S.SPH_FP64 if precision == "fp64" else S.SPH_MIXED
    lmax, nz, nlat, nphi = 31, 70, 48, 96
    P = O.Plan(lmax, nz, nlat=nlat, nphi=nphi, C=25, d=5)
    G = S.Plan(lmax, nz, nlat=nlat, nphi=nphi, Cz=25, oz=5, precision=prec)
    rng = np.random.default_rng(31)
    grid = dev(P.sh_synthesis(random_spec(P, rng)))
    qst = [dev(P.z_forward(random_spec(P, rng))) for _ in range(3)]

    # whole field
    carr_w = G.new_spec()
    S.fftp2d_real_to_complex_xy(G, grid, carr_w)
    spec_w = carr_w.clone()
    S.fftp1d_real_to_complex_z(G, spec_w)
    der_w, dlr_w = G.new_spec(), G.new_spec()
    S.derivr(G, carr_w, der_w, 1, "r")
    S.dlr(G, carr_w, dlr_w)
    syn_w = G.new_grid()
    S.fftp2d_complex_to_real_xy(G, carr_w, syn_w)
    vec_w = [G.new_grid() for _ in range(3)]
    S.fftp2d_qst_to_vec(G, *qst, *vec_w)

    # ranks: 2D on their planes, the exchange, z and operators on their lm columns
    planes = _ranges(S, nz, NPROCS)
    cols = _ranges(S, G.nlm, NPROCS)
    carr = torch.empty_like(carr_w)
    syn = torch.empty_like(syn_w)
    vec = [torch.empty_like(x) for x in vec_w]
    for k0, k1 in planes:
        S.set_slab(G, k0, k1 - k0 + 1, 0, G.nlm)
        out = G.new_plane_spec()
        S.fftp2d_real_to_complex_xy(G, grid[k0:k1 + 1].contiguous(), out)
        carr[k0:k1 + 1] = out
        g = G.new_grid()
        S.fftp2d_complex_to_real_xy(G, carr_w[k0:k1 + 1].contiguous(), g)
        syn[k0:k1 + 1] = g
        vg = [G.new_grid() for _ in range(3)]
        S.fftp2d_qst_to_vec(G, *(x[k0:k1 + 1].contiguous() for x in qst), *vg)
        for a, b in zip(vec, vg):
            a[k0:k1 + 1] = b
    assert torch.equal(carr, carr_w)
    assert torch.equal(syn, syn_w)
    for a, b in zip(vec, vec_w):
        assert torch.equal(a, b)
    for (k0, k1), (l0, l1) in zip(planes, cols):
        S.set_slab(G, k0, k1 - k0 + 1, l0, l1 - l0 + 1)
        mine = carr[:, l0:l1 + 1].contiguous()
        z = mine.clone()
        S.fftp1d_real_to_complex_z(G, z)
        assert torch.equal(z, spec_w[:, l0:l1 + 1])
        d, e = G.new_spec(), G.new_spec()
        S.derivr(G, mine, d, 1, "r")
        S.dlr(G, mine, e)
        assert torch.equal(d, der_w[:, l0:l1 + 1])
        assert torch.equal(e, dlr_w[:, l0:l1 + 1])
        # the 3D transform (which needs the slab transpose) refuses a slab
        rc = S.lib().sph_fftp3d_real_to_complex(G.h, ctypes.c_void_p(grid.data_ptr()),
                                                ctypes.c_void_p(spec_w.data_ptr()), None)
        assert rc == 1  # SPH_EINVAL
    S.set_slab(G, 0, nz, 0, G.nlm)
    G.close()


def test_slab_operators_and_boundary():
    from redondito_b200 import sphp as S
    lmax, nz = 15, 64
    P = O.Plan(lmax, nz, nlat=24, nphi=48, C=25, d=5, rint=0.5, rext=1.5)
    G = S.Plan(lmax, nz, nlat=24, nphi=48, Cz=25, oz=5, rint=0.5, rext=1.5)
    S.setup_bc(G)
    rng = np.random.default_rng(5)
    a, tor, phi = (dev(random_spec(P, rng)) for _ in range(3))
    whole = {}
    for name, fn in (("laplang", lambda x, y: S.laplang(G, x, y)), ("multr", lambda x, y: S.multr(G, x, y, -2)),
                     ("derivr2", lambda x, y: S.derivr(G, x, y, 2, "r")),
                     ("derivk", lambda x, y: S.derivr(G, x, y, 1, "k")), ("invDl", lambda x, y: S.invDl(G, x, y))):
        y = G.new_spec()
        fn(a, y)
        whole[name] = (fn, y)
    T_w, F_w, W_w = tor.clone(), phi.clone(), G.new_spec()
    S.v_imposebc(G, T_w, F_w, W_w)
    Tf_w, Ff_w, Wf_w = tor.clone(), phi.clone(), G.new_spec()
    S.v_imposebc_fast(G, Tf_w, Ff_w, Wf_w)
    x, y = a.clone(), G.new_spec()
    S.fc_filter(G, x, "r")
    S.saxpby_c(G, y, a, 2.0, x, -0.5)
    for l0, l1 in _ranges(S, G.nlm, 4):
        n = l1 - l0 + 1
        S.set_slab(G, 0, nz, l0, n)
        sl = slice(l0, l1 + 1)
        for name, (fn, yw) in whole.items():
            out = G.new_spec()
            fn(a[:, sl].contiguous(), out)
            assert torch.equal(out, yw[:, sl]), name
        T, F, W = tor[:, sl].contiguous(), phi[:, sl].contiguous(), G.new_spec()
        S.v_imposebc(G, T, F, W)
        assert torch.equal(T, T_w[:, sl]) and torch.equal(F, F_w[:, sl]) and torch.equal(W, W_w[:, sl])
        T, F, W = tor[:, sl].contiguous(), phi[:, sl].contiguous(), G.new_spec()
        S.v_imposebc_fast(G, T, F, W)
        assert torch.equal(F, Ff_w[:, sl]) and torch.equal(W, Wf_w[:, sl])
        xs = a[:, sl].contiguous()
        S.fc_filter(G, xs, "r")
        assert torch.equal(xs, x[:, sl])
        ys = G.new_spec()
        S.saxpby_c(G, ys, a[:, sl].contiguous(), 2.0, xs, -0.5)
        assert torch.equal(ys, y[:, sl])
    S.set_slab(G, 0, nz, 0, G.nlm)
    G.close()


def test_split_3d_pair_one_rank_over_nccl():
    """The split 3D transforms of redondito_b200/slab.py through an NCCL
    process group of one rank (the exchange moves every block to itself)
    equal the unsplit 3D transforms bit for bit.  Several ranks are covered
    on the CPU (tests/test_slab_gloo.py)."""
    import socket

    import torch.distributed as dist
    from redondito_b200 import slab, sphp as S
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        P = O.Plan(31, 64, nlat=48, nphi=96, C=25, d=5)
        G = S.Plan(31, 64, nlat=48, nphi=96, Cz=25, oz=5)
        grid = dev(P.sh_synthesis(random_spec(P, np.random.default_rng(8))))
        ref = G.new_spec()
        S.fftp3d_real_to_complex(G, grid, ref)
        spec = G.new_spec()
        slab.fftp3d_real_to_complex(G, grid, spec)
        assert torch.equal(spec, ref)
        g1, g2 = G.new_grid(), G.new_grid()
        S.set_slab(G, 0, G.nz, 0, G.nlm)
        S.fftp3d_complex_to_real(G, ref.clone(), g1)
        slab.fftp3d_complex_to_real(G, spec, g2)
        assert torch.equal(g1, g2)
        S.set_slab(G, 0, G.nz, 0, G.nlm)
        G.close()
    finally:
        dist.destroy_process_group()
