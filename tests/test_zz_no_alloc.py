"""The allocation-free radial derivative against the plan-based one.

sph_derivr_noalloc serves callers that cannot allocate device memory (their
device memory belongs to another allocator); it keeps its tables in one
file-scope device array that every call rewrites.  Calls in a row with
different sizes and orders must each match sph_derivr on the same input, so
a call cannot be reading tables left over from the one before.  Both paths
run the same kernel on tables built the same way, so they agree to a few
units in the last place (TOL_SAME).  The cases cover every order p = 1..4,
the compile-time FFT lengths and the generic one (nz = 200), the largest
transform (nz = 4096, one column per CTA) and the largest continuation
operator (Cz*oz = 2048).  A repeated call must leave the device's free
memory unchanged.  This file is collected last so that a failure here comes
after every other test.
"""
import ctypes

import numpy as np
import pytest

from tests._helpers import check, rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_SAME = 1e-14


def _call(lib, a, out, nlm, nz, C, d, rint, rext, dir_, order):
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dptr = (ctypes.c_double * len(dir_))(*dir_) if C > 0 else None
    return lib.sph_derivr_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                  nlm, nz, C, d, rint, rext, dptr, order, stream)


def _one(S, lib, lmax, nz, order, seed, C=25, d=5, dir_=None):
    rint, rext = 0.35, 1.0
    if C > 0 and dir_ is None:
        dir_ = S.load_dirichlet_tables(C, d)
    P = S.Plan(lmax, nz, Cz=C, oz=d, rint=rint, rext=rext, dir=dir_)
    rng = np.random.default_rng(seed)
    a_h = rng.normal(size=(nz, P.nlm)) + 1j * rng.normal(size=(nz, P.nlm))
    a = torch.from_numpy(a_h).cuda()
    ref = P.new_spec()
    S.derivr(P, a, ref, order, "r")
    out = torch.full_like(ref, float("nan"))
    assert _call(lib, a, out, P.nlm, nz, C, d, rint, rext, dir_, order) == 0
    torch.cuda.synchronize()
    assert torch.isfinite(out).all()
    check(rel_l2(out.cpu().numpy(), ref.cpu().numpy()), TOL_SAME, f"nz={nz} p={order} Cz*oz={C * d}")
    P.close()


def test_noalloc_derivative_matches_plan_path_twice():
    from redondito_b200 import sphp as S
    lib = S.lib()
    _one(S, lib, 31, 128, 1, 1)
    _one(S, lib, 15, 96, 2, 2)


def test_noalloc_orders_and_lengths():
    """p = 3 and 4; a length outside the compile-time FFT set; the largest
    transform; the largest continuation operator (a seeded stand-in with
    Cz = 64, oz = 32: the kernel applies whatever operator it is given)."""
    from redondito_b200 import sphp as S
    lib = S.lib()
    _one(S, lib, 7, 64, 3, 3)
    _one(S, lib, 7, 128, 4, 4)
    _one(S, lib, 15, 200, 1, 5)
    _one(S, lib, 3, 4096, 2, 6)
    rng = np.random.default_rng(7)
    big = list(rng.normal(size=64 * 32) / 32.0)
    _one(S, lib, 3, 4096, 1, 8, C=64, d=32, dir_=big)


def test_noalloc_leaves_device_memory_unchanged():
    """A call after the first one on a device (which looks up the array's
    address and loads the kernel) allocates nothing: the device's free
    memory and torch's allocator are the same before and after it."""
    from redondito_b200 import sphp as S
    lib = S.lib()
    C, d, nz, nlm = 25, 5, 256, 4096
    dir_ = S.load_dirichlet_tables(C, d)
    a = torch.randn((nz, nlm), dtype=torch.complex128, device="cuda")
    out = torch.empty_like(a)
    assert _call(lib, a, out, nlm, nz, C, d, 0.35, 1.0, dir_, 1) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for order in (1, 2):
        assert _call(lib, a, out, nlm, nz, C, d, 0.35, 1.0, dir_, order) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_rejects_oversize():
    from redondito_b200 import sphp as S
    lib = S.lib()
    x = torch.zeros((8192, 4), dtype=torch.complex128, device="cuda")
    rc = lib.sph_derivr_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                4, 8192, 0, 0, 0.0, 1.0, None, 1, None)
    assert rc == 1  # SPH_EINVAL: nz beyond the 4096 limit
    dir_ = (ctypes.c_double * (64 * 33))()
    rc = lib.sph_derivr_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                4, 4096, 64, 33, 0.0, 1.0, dir_, 1, None)
    assert rc == 1  # SPH_EINVAL: Cz*oz beyond the 2048 limit
    rc = lib.sph_derivr_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                4, 64, 0, 0, 0.0, 1.0, None, 5, None)
    assert rc == 1  # SPH_EINVAL: order beyond 4
