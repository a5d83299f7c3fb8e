"""The allocation-free radial derivative against the plan-based one.

sph_derivr_noalloc serves callers that cannot allocate device memory (their
device memory belongs to another allocator); it keeps its tables in one
file-scope device array that every call rewrites.  Two calls in a row with
different sizes and orders must each match sph_derivr on the same input, so
the second call cannot be reading tables left over from the first.  This
file is collected last so that a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

from tests._helpers import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL_CONT = 1e-11   # the tolerance of the other FC-Gram derivative tests
TOL_D2 = 1e-10


def _one(S, lib, lmax, nz, order, seed):
    C, d, rint, rext = 25, 5, 0.35, 1.0
    P = S.Plan(lmax, nz, Cz=C, oz=d, rint=rint, rext=rext)
    rng = np.random.default_rng(seed)
    a_h = rng.normal(size=(nz, P.nlm)) + 1j * rng.normal(size=(nz, P.nlm))
    a = torch.from_numpy(a_h).cuda()
    ref = P.new_spec()
    S.derivr(P, a, ref, order, "r")
    out = torch.full_like(ref, float("nan"))
    dir_ = (ctypes.c_double * (C * d))(*S.load_dirichlet_tables(C, d))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.sph_derivr_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                P.nlm, nz, C, d, rint, rext, dir_, order, stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert torch.isfinite(out).all()
    tol = TOL_CONT if order == 1 else TOL_D2
    assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) < tol
    P.close()


def test_noalloc_derivative_matches_plan_path_twice():
    from redondito_b200 import sphp as S
    lib = S.lib()
    _one(S, lib, 31, 128, 1, 1)
    _one(S, lib, 15, 96, 2, 2)


def test_noalloc_rejects_oversize():
    from redondito_b200 import sphp as S
    lib = S.lib()
    x = torch.zeros((8192, 4), dtype=torch.complex128, device="cuda")
    rc = lib.sph_derivr_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                4, 8192, 0, 0, 0.0, 1.0, None, 1, None)
    assert rc == 1  # SPH_EINVAL: nz beyond the 4096 limit
