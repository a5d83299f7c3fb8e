"""Host-side mirror of REDONDITO's sphp / pseudo / boundary interfaces over
the B200 C ABI (include/sph_b200.h, redondito_b200/_lib/libsph_b200.so).

The names and argument meanings follow the reference's Fortran routines
(src/sphp-gpu/sphp_sca.F90, src/sphp-gpu/sphp_vec.F90,
src/pseudo/pseudospec_hd.f90, src/boundary/*.f90) so that code written
against them reads the same:

    plan = Plan(lmax=31, nz=58, Cz=25, oz=5, rint=0.35, rext=1.0)
    fftp3d_real_to_complex(plan, grid, spec)      # grid (nz,nphi,nlat) f64
    fftp3d_complex_to_real(plan, spec, grid)      # spec (nz,nlm) c128, destroyed
    derivr(plan, a, b, 1, 'r')

Fields are torch tensors on the plan's CUDA device: physical fields float64
of shape (nz, nphi, nlat) (Fortran f(nlat,nphi,nz)), spectral fields
complex128 of shape (nz, nlm) (Fortran f(nlm,nz)).  PyTorch only provides
device memory and the current stream; every transform runs in the sm_100a
library.  There is no CPU fallback: without the built library or a CUDA
device the calls raise.

Errors: the reference prints and STOPs (e.g. fcgram_mod.f90:96-102); here a
non-zero status from the library raises SphError with the code's name.
"""
import ctypes
import os

import torch

from . import build as _build

SPH_FP64, SPH_MIXED = 0, 1
_CODES = {1: "SPH_EINVAL", 2: "SPH_ENOMEM", 3: "SPH_ECUDA", 4: "SPH_ENOTREADY", 5: "SPH_EIO",
          6: "SPH_ETIMEDOUT"}
TABLES_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tables")

# exported symbols, as declared in include/sph_b200.h
SYMBOLS = (
    "sph_plan_create", "sph_plan_destroy", "sph_fcgram_load_tables", "sph_plan_sizes", "sph_grid",
    "sph_fftp2d_real_to_complex_xy", "sph_fftp2d_complex_to_real_xy",
    "sph_fftp1d_real_to_complex_z", "sph_fftp1d_complex_to_real_z",
    "sph_fftp3d_real_to_complex", "sph_fftp3d_complex_to_real",
    "sph_fftp2d_vec_to_qst", "sph_fftp2d_qst_to_vec",
    "sph_derivr", "sph_laplang", "sph_multr", "sph_dlr", "sph_saxpby_c", "sph_saxpby_r",
    "sph_fc_filter", "sph_copy", "sph_prodvec",
    "sph_setup_bc", "sph_dirichlet", "sph_invDl", "sph_v_imposebc", "sph_v_imposebc_fast",
    "sph_nl_rhs", "sph_rk3_step",
    "sph_timer_enable", "sph_timer_reset", "sph_timer_read",
    "sph_derivr_noalloc", "sph_plan_status", "sph_fftp3d_vec_to_qst", "sph_fftp3d_qst_to_vec",
    "sph_batch_create", "sph_batch_run", "sph_batch_status", "sph_batch_destroy",
    "sph_plan_set_tiles", "sph_plan_set_slab", "sph_range",
    "sph_read_namelist", "sph_write_grids", "sph_energy_spectrum", "sph_run", "sph_plan_clone",
    "sph_fcgram_load_neumann_tables", "sph_plan_set_neumann", "sph_neumann_reconstruct",
    "sph_robin_reconstruct",
    "sph_fftp2d_real_to_complex_xy_f32", "sph_fftp2d_complex_to_real_xy_f32",
    "sph_fftp1d_real_to_complex_z_f32", "sph_fftp1d_complex_to_real_z_f32",
    "sph_fftp3d_real_to_complex_f32", "sph_fftp3d_complex_to_real_f32",
    "sph_fftp2d_vec_to_qst_f32", "sph_fftp2d_qst_to_vec_f32",
    "sph_fftp3d_vec_to_qst_f32", "sph_fftp3d_qst_to_vec_f32",
    "sph_derivr_f32", "sph_dlr_f32", "sph_fc_filter_f32",
    "sph_laplang_f32", "sph_multr_f32", "sph_saxpby_c_f32", "sph_saxpby_r_f32", "sph_copy_f32",
    "sph_prodvec_f32", "sph_dirichlet_f32", "sph_invDl_f32", "sph_v_imposebc_f32",
    "sph_v_imposebc_fast_f32", "sph_nl_rhs_f32", "sph_rk3_step_f32",
)
TIMER_CLASSES = ("phi_fwd", "phi_inv", "leg_analysis", "leg_synthesis", "vec_analysis",
                 "vec_synthesis", "zfft", "ops")


class SphError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__(f"{fn} failed: {_CODES.get(code, code)}")
        self.code = code


_lib = None


def lib(build_if_missing=True):
    """Load the in-tree library (building it with nvcc if it is stale)."""
    global _lib
    if _lib is None:
        if build_if_missing and not _build.up_to_date():
            _build.build()
        if not os.path.exists(_build.LIB):
            raise RuntimeError(f"{_build.LIB} is not built; run python -m redondito_b200.build")
        L = ctypes.CDLL(_build.LIB)
        P, I, D, Vp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p
        pD = ctypes.POINTER(ctypes.c_double)
        pI = ctypes.POINTER(ctypes.c_int)
        sig = {
            "sph_plan_create": [ctypes.POINTER(P), I, I, I, I, I, I, D, D, pD, I],
            "sph_plan_destroy": [P],
            "sph_fcgram_load_tables": [ctypes.c_char_p, I, I, pD],
            "sph_plan_sizes": [P, pI, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)],
            "sph_grid": [P, pD, pD, pD, pD, pD, pI, pI],
            "sph_fftp2d_real_to_complex_xy": [P, Vp, Vp, Vp],
            "sph_fftp2d_complex_to_real_xy": [P, Vp, Vp, Vp],
            "sph_fftp1d_real_to_complex_z": [P, Vp, Vp],
            "sph_fftp1d_complex_to_real_z": [P, Vp, Vp],
            "sph_fftp3d_real_to_complex": [P, Vp, Vp, Vp],
            "sph_fftp3d_complex_to_real": [P, Vp, Vp, Vp],
            "sph_fftp2d_vec_to_qst": [P] + [Vp] * 6 + [Vp],
            "sph_fftp2d_qst_to_vec": [P] + [Vp] * 6 + [Vp],
            "sph_derivr": [P, Vp, Vp, I, ctypes.c_char, Vp],
            "sph_laplang": [P, Vp, Vp, Vp],
            "sph_multr": [P, Vp, Vp, I, Vp],
            "sph_dlr": [P, Vp, Vp, Vp],
            "sph_saxpby_c": [P, Vp, Vp, D, Vp, D, Vp],
            "sph_saxpby_r": [P, Vp, Vp, D, Vp, D, Vp],
            "sph_fc_filter": [P, Vp, ctypes.c_char, Vp],
            "sph_copy": [P, Vp, Vp, Vp],
            "sph_prodvec": [P] + [Vp] * 9 + [Vp],
            "sph_setup_bc": [P, ctypes.c_char_p, ctypes.c_char_p],
            "sph_dirichlet": [P, Vp, Vp],
            "sph_invDl": [P, Vp, Vp, Vp],
            "sph_v_imposebc": [P, Vp, Vp, Vp, Vp],
            "sph_v_imposebc_fast": [P, Vp, Vp, Vp, Vp],
            "sph_nl_rhs": [P, Vp, Vp, Vp, D, Vp, Vp, pD, Vp],
            "sph_rk3_step": [P, Vp, Vp, Vp, D, D, pD, Vp],
            "sph_timer_enable": [P, I],
            "sph_timer_reset": [P],
            "sph_timer_read": [P, pD, pI],
            "sph_derivr_noalloc": [Vp, Vp, I, I, I, I, D, D, pD, I, Vp],
            "sph_plan_status": [P],
            "sph_fftp3d_vec_to_qst": [P] + [Vp] * 6 + [Vp],
            "sph_fftp3d_qst_to_vec": [P] + [Vp] * 6 + [Vp],
            "sph_batch_create": [ctypes.POINTER(P), I, ctypes.POINTER(P), pI, ctypes.POINTER(P),
                                 ctypes.POINTER(P), ctypes.POINTER(P)],
            "sph_batch_run": [P, Vp],
            "sph_batch_status": [P],
            "sph_batch_destroy": [P],
            "sph_plan_set_tiles": [P, I, I, I],
            "sph_plan_set_slab": [P, I, I, I, I],
            "sph_range": [I, I, I, I, pI, pI],
            "sph_read_namelist": [ctypes.c_char_p, pI, pI, pI, pI, pD, pD, pD, pI, pI, pI, pD, pI],
            "sph_write_grids": [P, ctypes.c_char_p],
            "sph_energy_spectrum": [P, Vp, Vp, pD, Vp],
            "sph_run": [P, Vp, Vp, Vp, D, D, I, I, I, I, ctypes.c_char_p, pD, Vp],
            "sph_plan_clone": [P, ctypes.POINTER(P)],
            "sph_fcgram_load_neumann_tables": [ctypes.c_char_p, I, I, D, pD],
            "sph_plan_set_neumann": [P, pD, pD],
            "sph_neumann_reconstruct": [P, Vp, I, I, Vp],
            "sph_robin_reconstruct": [P, Vp, I, Vp, Vp],
            "sph_fftp2d_real_to_complex_xy_f32": [P, Vp, Vp, Vp],
            "sph_fftp2d_complex_to_real_xy_f32": [P, Vp, Vp, Vp],
            "sph_fftp1d_real_to_complex_z_f32": [P, Vp, Vp],
            "sph_fftp1d_complex_to_real_z_f32": [P, Vp, Vp],
            "sph_fftp3d_real_to_complex_f32": [P, Vp, Vp, Vp],
            "sph_fftp3d_complex_to_real_f32": [P, Vp, Vp, Vp],
            "sph_fftp2d_vec_to_qst_f32": [P] + [Vp] * 6 + [Vp],
            "sph_fftp2d_qst_to_vec_f32": [P] + [Vp] * 6 + [Vp],
            "sph_fftp3d_vec_to_qst_f32": [P] + [Vp] * 6 + [Vp],
            "sph_fftp3d_qst_to_vec_f32": [P] + [Vp] * 6 + [Vp],
            "sph_derivr_f32": [P, Vp, Vp, I, ctypes.c_char, Vp],
            "sph_dlr_f32": [P, Vp, Vp, Vp],
            "sph_fc_filter_f32": [P, Vp, ctypes.c_char, Vp],
            "sph_laplang_f32": [P, Vp, Vp, Vp],
            "sph_multr_f32": [P, Vp, Vp, I, Vp],
            "sph_saxpby_c_f32": [P, Vp, Vp, D, Vp, D, Vp],
            "sph_saxpby_r_f32": [P, Vp, Vp, D, Vp, D, Vp],
            "sph_copy_f32": [P, Vp, Vp, Vp],
            "sph_prodvec_f32": [P] + [Vp] * 9 + [Vp],
            "sph_dirichlet_f32": [P, Vp, Vp],
            "sph_invDl_f32": [P, Vp, Vp, Vp],
            "sph_v_imposebc_f32": [P, Vp, Vp, Vp, Vp],
            "sph_v_imposebc_fast_f32": [P, Vp, Vp, Vp, Vp],
            "sph_nl_rhs_f32": [P, Vp, Vp, Vp, D, Vp, Vp, pD, Vp],
            "sph_rk3_step_f32": [P, Vp, Vp, Vp, D, D, pD, Vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        _lib = L
    return _lib


def _check(fn, rc):
    if rc != 0:
        raise SphError(fn, rc)


def _call(name, *args):
    _check(name, getattr(lib(), name)(*args))


def nlat_for(lmax):
    """grid_init rule (src/pseudo/pseudospec_mod.f90:67)."""
    return 4 * ((3 * (lmax + 1) + 7) // 8)


def load_dirichlet_tables(C=25, d=5, tdir=TABLES_DIR):
    """load_dirichlet_tables (src/sphp/fcgram_mod.f90:186-263): dir = A.Q^T."""
    out = (ctypes.c_double * (C * d))()
    _call("sph_fcgram_load_tables", tdir.encode(), C, d, out)
    return list(out)


def load_neumann_tables(d=5, ord=1, dx=1.0, tdir=TABLES_DIR):
    """load_neumann_tables (src/sphp/fcgram_mod.f90:267-365): the boundary
    reconstructor from the ord-th normal derivative, scaled for grid step dx."""
    out = (ctypes.c_double * d)()
    _call("sph_fcgram_load_neumann_tables", tdir.encode(), int(d), int(ord), float(dx), out)
    return list(out)


class Plan:
    """fcgram_create_plan + grid_init/box_init: the angular grid, the FC-Gram
    continuation in z, the device tables and the plan's scratch."""

    def __init__(self, lmax, nz, nlat=None, nphi=None, Cz=0, oz=0, rint=0.35, rext=1.0,
                 tdir=TABLES_DIR, precision=SPH_FP64, device=None, dir=None):
        """dir: the Cz x oz continuation operator, column-major (Cz*oz
        values); by default it is read from the FC-Gram tables in tdir."""
        if not torch.cuda.is_available():
            raise RuntimeError("redondito_b200 needs a CUDA device (B200, sm_100a)")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.lmax, self.nz, self.Cz, self.oz = lmax, nz, Cz, oz
        self.nlat = nlat if nlat is not None else nlat_for(lmax)
        self.nphi = nphi if nphi is not None else 2 * self.nlat
        self.rint, self.rext = rint, rext
        self.precision = precision
        dirp = None
        if Cz > 0:
            d = load_dirichlet_tables(Cz, oz, tdir) if dir is None else [float(x) for x in dir]
            if len(d) != Cz * oz:
                raise ValueError(f"dir must hold Cz*oz = {Cz * oz} values")
            self._dir = (ctypes.c_double * len(d))(*d)
            dirp = self._dir
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _call("sph_plan_create", ctypes.byref(h), lmax, self.nlat, self.nphi, nz, Cz, oz,
                  float(rint), float(rext), dirp, int(precision))
        self.h = h
        self.nlm = (lmax + 1) * (lmax + 2) // 2
        self.N = nz - Cz
        self.k0, self.nzv, self.lm0, self.nlmv = 0, nz, 0, self.nlm
        self.dz = (rext - rint) / (nz - Cz - 1) if nz - Cz > 1 else 1.0
        if Cz > 0 and os.path.exists(os.path.join(tdir, f"Q1n{oz}.dat")):
            # the Neumann reconstructors (fcgram_mod.f90:267-365), for the freeslip walls
            n1 = (ctypes.c_double * oz)(*load_neumann_tables(oz, 1, self.dz, tdir))
            n2 = (ctypes.c_double * oz)(*load_neumann_tables(oz, 2, self.dz, tdir))
            _call("sph_plan_set_neumann", self.h, n1, n2)
        self._grid_arrays()
        self._bc = False

    def clone(self):
        """A plan of the same sizes sharing this plan's device tables, with
        scratch of its own (sph_plan_clone)."""
        c = object.__new__(Plan)
        c.__dict__.update({k: v for k, v in self.__dict__.items() if k not in ("h", "_bc")})
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _call("sph_plan_clone", self.h, ctypes.byref(h))
        c.h = h
        c._bc = False
        c.k0, c.nzv, c.lm0, c.nlmv = 0, self.nz, 0, self.nlm
        return c

    def _grid_arrays(self):
        def dbl(n):
            return (ctypes.c_double * n)()
        th, w, ph, z, kz = dbl(self.nlat), dbl(self.nlat), dbl(self.nphi), dbl(self.nz), dbl(self.nz)
        ell, emm = (ctypes.c_int * self.nlm)(), (ctypes.c_int * self.nlm)()
        _call("sph_grid", self.h, th, w, ph, z, kz, ell, emm)
        self.theta = torch.tensor(list(th), dtype=torch.float64)
        self.weights = torch.tensor(list(w), dtype=torch.float64)
        self.phi = torch.tensor(list(ph), dtype=torch.float64)
        self.z = torch.tensor(list(z), dtype=torch.float64)
        self.kz = torch.tensor(list(kz), dtype=torch.float64)
        self.ell = torch.tensor(list(ell), dtype=torch.int32)
        self.emm = torch.tensor(list(emm), dtype=torch.int32)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().sph_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # allocation helpers (the caller's slab: see set_slab)
    def new_grid(self):
        return torch.zeros((self.nzv, self.nphi, self.nlat), dtype=torch.float64, device=self.device)

    def new_spec(self):
        return torch.zeros((self.nz, self.nlmv), dtype=torch.complex128, device=self.device)

    def new_grid32(self):
        """a float grid for the single-precision entry points (whole field)"""
        return torch.zeros((self.nz, self.nphi, self.nlat), dtype=torch.float32, device=self.device)

    def new_spec32(self):
        """float complex spectra for the single-precision entry points (whole field)"""
        return torch.zeros((self.nz, self.nlm), dtype=torch.complex64, device=self.device)

    def new_plane_spec(self):
        """per-plane spectra of the caller's planes, (nplanes, nlm)"""
        return torch.zeros((self.nzv, self.nlm), dtype=torch.complex128, device=self.device)

    def lm(self, l, m):
        return m * (2 * self.lmax + 1 - m) // 2 + l


def _ptr(t, shape, dtype):
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise TypeError("fields must be CUDA tensors")
    if t.dtype != dtype or tuple(t.shape) != tuple(shape) or not t.is_contiguous():
        raise ValueError(f"expected contiguous {dtype} tensor of shape {tuple(shape)}, "
                         f"got {t.dtype} {tuple(t.shape)}")
    return ctypes.c_void_p(t.data_ptr())


def _g(plan, t):
    """physical array of the caller's planes: (nplanes, nphi, nlat)"""
    return _ptr(t, (plan.nzv, plan.nphi, plan.nlat), torch.float64)


def _s(plan, t):
    """spectral array of the caller's lm columns: (nz, nlm_local)"""
    return _ptr(t, (plan.nz, plan.nlmv), torch.complex128)


def _sp(plan, t):
    """per-plane spectra of the caller's planes (the 2D transforms): (nplanes, nlm)"""
    return _ptr(t, (plan.nzv, plan.nlm), torch.complex128)


def _g32(plan, t):
    """float grid of the whole field (single-precision entry points)"""
    return _ptr(t, (plan.nz, plan.nphi, plan.nlat), torch.float32)


def _s32(plan, t):
    """float complex spectra of the whole field (single-precision entry points)"""
    return _ptr(t, (plan.nz, plan.nlm), torch.complex64)


def set_slab(plan, k0, nplanes, lm0, nlm_local):
    """The caller's slab (see sph_plan_set_slab): planes [k0, k0+nplanes) for
    the 2D transforms, lm columns [lm0, lm0+nlm_local) for the z transforms,
    operators and boundary.  set_slab(plan, 0, nz, 0, nlm) restores the
    whole field."""
    _call("sph_plan_set_slab", plan.h, int(k0), int(nplanes), int(lm0), int(nlm_local))
    plan.k0, plan.nzv, plan.lm0, plan.nlmv = int(k0), int(nplanes), int(lm0), int(nlm_local)


def range_(n1, n2, nprocs, irank):
    """range (src/sphp/sphp_sca.F90:596-626): (ista, iend), inclusive."""
    a, b = ctypes.c_int(), ctypes.c_int()
    _call("sph_range", int(n1), int(n2), int(nprocs), int(irank), ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


# ---------------------------------------------------------------- transforms
def fftp2d_real_to_complex_xy(plan, in_, out, stream=None):
    _call("sph_fftp2d_real_to_complex_xy", plan.h, _g(plan, in_), _sp(plan, out), _stream(stream))


def fftp2d_complex_to_real_xy(plan, in_, out, stream=None):
    _call("sph_fftp2d_complex_to_real_xy", plan.h, _sp(plan, in_), _g(plan, out), _stream(stream))


def fftp1d_real_to_complex_z(plan, inout, stream=None):
    _call("sph_fftp1d_real_to_complex_z", plan.h, _s(plan, inout), _stream(stream))


def fftp1d_complex_to_real_z(plan, inout, stream=None):
    _call("sph_fftp1d_complex_to_real_z", plan.h, _s(plan, inout), _stream(stream))


def fftp3d_real_to_complex(plan, in_, out, stream=None):
    _call("sph_fftp3d_real_to_complex", plan.h, _g(plan, in_), _s(plan, out), _stream(stream))


def fftp3d_complex_to_real(plan, in_, out, stream=None):
    """The input may be destroyed, as in the reference (FP64 plans transform it
    in place in z; mixed plans write the z inverse into the synthesis tiles)."""
    _call("sph_fftp3d_complex_to_real", plan.h, _s(plan, in_), _g(plan, out), _stream(stream))


def fftp2d_vec_to_qst(plan, vr, vt, vp, q, s, t, stream=None):
    _call("sph_fftp2d_vec_to_qst", plan.h, _g(plan, vr), _g(plan, vt), _g(plan, vp),
          _sp(plan, q), _sp(plan, s), _sp(plan, t), _stream(stream))


def fftp2d_qst_to_vec(plan, q, s, t, vr, vt, vp, stream=None):
    _call("sph_fftp2d_qst_to_vec", plan.h, _sp(plan, q), _sp(plan, s), _sp(plan, t),
          _g(plan, vr), _g(plan, vt), _g(plan, vp), _stream(stream))


def fftp3d_vec_to_qst(plan, vr, vt, vp, q, s, t, stream=None):
    """fftp2d_vec_to_qst followed by the z transform of q, s and t."""
    _call("sph_fftp3d_vec_to_qst", plan.h, _g(plan, vr), _g(plan, vt), _g(plan, vp),
          _s(plan, q), _s(plan, s), _s(plan, t), _stream(stream))


def fftp3d_qst_to_vec(plan, q, s, t, vr, vt, vp, stream=None):
    """Inverse z transform of q, s, t (in place), then fftp2d_qst_to_vec."""
    _call("sph_fftp3d_qst_to_vec", plan.h, _s(plan, q), _s(plan, s), _s(plan, t),
          _g(plan, vr), _g(plan, vt), _g(plan, vp), _stream(stream))


# ---------------------------------------------------------------- operators
def derivr(plan, a, b, p, esp, stream=None):
    _call("sph_derivr", plan.h, _s(plan, a), _s(plan, b), int(p), esp.encode()[:1], _stream(stream))


def derivr_noalloc(a, b, nz, Cz, oz, rint, rext, dir, p, stream=None):
    """Radial derivative without a plan and without allocation (see
    sph_derivr_noalloc in include/sph_b200.h); a, b complex128 (nz, nlm)."""
    nlm = a.shape[1]
    if tuple(b.shape) != tuple(a.shape) or a.shape[0] != nz:
        raise ValueError("a and b must both be (nz, nlm)")
    d = None
    if Cz > 0:
        d = (ctypes.c_double * (Cz * oz))(*dir)
    _call("sph_derivr_noalloc", ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), nlm, nz,
          Cz, oz, float(rint), float(rext), d, int(p), _stream(stream))


def laplang(plan, a, b, stream=None):
    _call("sph_laplang", plan.h, _s(plan, a), _s(plan, b), _stream(stream))


def multr(plan, a, b, p, stream=None):
    _call("sph_multr", plan.h, _s(plan, a), _s(plan, b), int(p), _stream(stream))


def dlr(plan, a, b, stream=None):
    _call("sph_dlr", plan.h, _s(plan, a), _s(plan, b), _stream(stream))


def saxpby_c(plan, z, x, a, y, b, stream=None):
    _call("sph_saxpby_c", plan.h, _s(plan, z), _s(plan, x), float(a), _s(plan, y), float(b),
          _stream(stream))


def saxpby_r(plan, z, x, a, y, b, stream=None):
    _call("sph_saxpby_r", plan.h, _g(plan, z), _g(plan, x), float(a), _g(plan, y), float(b),
          _stream(stream))


def fc_filter(plan, a, esp, stream=None):
    _call("sph_fc_filter", plan.h, _s(plan, a), esp.encode()[:1], _stream(stream))


def copy(plan, a, b, stream=None):
    _call("sph_copy", plan.h, _s(plan, a), _s(plan, b), _stream(stream))


def prodvec(plan, ar, at, ap, br, bt, bp, cr, ct, cp, stream=None):
    _call("sph_prodvec", plan.h, *[_g(plan, x) for x in (ar, at, ap, br, bt, bp, cr, ct, cp)],
          _stream(stream))


# ---------------------------------------------------------------- boundary
def setup_bc(plan, bckind=("noslip", "noslip")):
    _call("sph_setup_bc", plan.h, bckind[0].encode(), bckind[1].encode())
    plan._bc = True


def neumann_reconstruct(plan, f, boun, ord=1, stream=None):
    """The wall row of f (boun 0 inner, 1 outer) from the ord-th outward
    normal derivative it holds (fcgram_mod.f90:368-520)."""
    _call("sph_neumann_reconstruct", plan.h, _s(plan, f), int(boun), int(ord), _stream(stream))


def robin_reconstruct(plan, f, boun, a, stream=None):
    """f' + a f = g at the wall (g in the wall row); a: float64 CUDA tensor of
    nlm coefficients (fcgram_mod.f90:523-650)."""
    if a.dtype != torch.float64 or a.device.type != "cuda" or a.numel() != plan.nlmv or not a.is_contiguous():
        raise ValueError("a must be a contiguous float64 CUDA tensor of nlm values")
    _call("sph_robin_reconstruct", plan.h, _s(plan, f), int(boun), ctypes.c_void_p(a.data_ptr()), _stream(stream))


def dirichlet(plan, a, stream=None):
    _call("sph_dirichlet", plan.h, _s(plan, a), _stream(stream))


def invDl(plan, a, b, stream=None):
    _call("sph_invDl", plan.h, _s(plan, a), _s(plan, b), _stream(stream))


def v_imposebc(plan, tor, phi, pol, stream=None):
    _call("sph_v_imposebc", plan.h, _s(plan, tor), _s(plan, phi), _s(plan, pol), _stream(stream))


def v_imposebc_fast(plan, tor, phi, pol, stream=None):
    _call("sph_v_imposebc_fast", plan.h, _s(plan, tor), _s(plan, phi), _s(plan, pol), _stream(stream))


# ---------------------------------------------------------------- single precision
# The arrays of a GSINGLE_PRECISION build of the reference
# (src/sphp/fprecision_mod.F90:13-18): float grids and complex64 spectra on
# an SPH_MIXED plan over whole fields; the inverse transforms preserve their
# input.
def fftp2d_real_to_complex_xy_f32(plan, in_, out, stream=None):
    _call("sph_fftp2d_real_to_complex_xy_f32", plan.h, _g32(plan, in_), _s32(plan, out), _stream(stream))


def fftp2d_complex_to_real_xy_f32(plan, in_, out, stream=None):
    _call("sph_fftp2d_complex_to_real_xy_f32", plan.h, _s32(plan, in_), _g32(plan, out), _stream(stream))


def fftp1d_real_to_complex_z_f32(plan, inout, stream=None):
    _call("sph_fftp1d_real_to_complex_z_f32", plan.h, _s32(plan, inout), _stream(stream))


def fftp1d_complex_to_real_z_f32(plan, inout, stream=None):
    _call("sph_fftp1d_complex_to_real_z_f32", plan.h, _s32(plan, inout), _stream(stream))


def fftp3d_real_to_complex_f32(plan, in_, out, stream=None):
    _call("sph_fftp3d_real_to_complex_f32", plan.h, _g32(plan, in_), _s32(plan, out), _stream(stream))


def fftp3d_complex_to_real_f32(plan, in_, out, stream=None):
    _call("sph_fftp3d_complex_to_real_f32", plan.h, _s32(plan, in_), _g32(plan, out), _stream(stream))


def fftp2d_vec_to_qst_f32(plan, vr, vt, vp, q, s, t, stream=None):
    _call("sph_fftp2d_vec_to_qst_f32", plan.h, _g32(plan, vr), _g32(plan, vt), _g32(plan, vp),
          _s32(plan, q), _s32(plan, s), _s32(plan, t), _stream(stream))


def fftp2d_qst_to_vec_f32(plan, q, s, t, vr, vt, vp, stream=None):
    _call("sph_fftp2d_qst_to_vec_f32", plan.h, _s32(plan, q), _s32(plan, s), _s32(plan, t),
          _g32(plan, vr), _g32(plan, vt), _g32(plan, vp), _stream(stream))


def fftp3d_vec_to_qst_f32(plan, vr, vt, vp, q, s, t, stream=None):
    _call("sph_fftp3d_vec_to_qst_f32", plan.h, _g32(plan, vr), _g32(plan, vt), _g32(plan, vp),
          _s32(plan, q), _s32(plan, s), _s32(plan, t), _stream(stream))


def fftp3d_qst_to_vec_f32(plan, q, s, t, vr, vt, vp, stream=None):
    _call("sph_fftp3d_qst_to_vec_f32", plan.h, _s32(plan, q), _s32(plan, s), _s32(plan, t),
          _g32(plan, vr), _g32(plan, vt), _g32(plan, vp), _stream(stream))


def derivr_f32(plan, a, b, order, esp="r", stream=None):
    _call("sph_derivr_f32", plan.h, _s32(plan, a), _s32(plan, b), int(order), esp.encode(), _stream(stream))


def dlr_f32(plan, a, b, stream=None):
    _call("sph_dlr_f32", plan.h, _s32(plan, a), _s32(plan, b), _stream(stream))


def fc_filter_f32(plan, a, esp="r", stream=None):
    _call("sph_fc_filter_f32", plan.h, _s32(plan, a), esp.encode(), _stream(stream))


def laplang_f32(plan, a, b, stream=None):
    _call("sph_laplang_f32", plan.h, _s32(plan, a), _s32(plan, b), _stream(stream))


def multr_f32(plan, a, b, p, stream=None):
    _call("sph_multr_f32", plan.h, _s32(plan, a), _s32(plan, b), int(p), _stream(stream))


def saxpby_c_f32(plan, z, x, a, y, b, stream=None):
    _call("sph_saxpby_c_f32", plan.h, _s32(plan, z), _s32(plan, x), float(a), _s32(plan, y), float(b),
          _stream(stream))


def saxpby_r_f32(plan, z, x, a, y, b, stream=None):
    _call("sph_saxpby_r_f32", plan.h, _g32(plan, z), _g32(plan, x), float(a), _g32(plan, y), float(b),
          _stream(stream))


def copy_f32(plan, a, b, stream=None):
    _call("sph_copy_f32", plan.h, _s32(plan, a), _s32(plan, b), _stream(stream))


def prodvec_f32(plan, ar, at, ap, br, bt, bp, cr, ct, cp, stream=None):
    _call("sph_prodvec_f32", plan.h, *[_g32(plan, x) for x in (ar, at, ap, br, bt, bp, cr, ct, cp)],
          _stream(stream))


def dirichlet_f32(plan, a, stream=None):
    _call("sph_dirichlet_f32", plan.h, _s32(plan, a), _stream(stream))


def invDl_f32(plan, phi, w, stream=None):
    _call("sph_invDl_f32", plan.h, _s32(plan, phi), _s32(plan, w), _stream(stream))


def v_imposebc_f32(plan, tor, phi, pol, stream=None):
    _call("sph_v_imposebc_f32", plan.h, _s32(plan, tor), _s32(plan, phi), _s32(plan, pol), _stream(stream))


def v_imposebc_fast_f32(plan, tor, phi, pol, stream=None):
    _call("sph_v_imposebc_fast_f32", plan.h, _s32(plan, tor), _s32(plan, phi), _s32(plan, pol), _stream(stream))


def nl_rhs_f32(plan, Z, W, phi, nu, rhs_z, rhs_phi, stream=None):
    e = ctypes.c_double(0.0)
    _call("sph_nl_rhs_f32", plan.h, _s32(plan, Z), _s32(plan, W), _s32(plan, phi), float(nu),
          _s32(plan, rhs_z), _s32(plan, rhs_phi), ctypes.byref(e), _stream(stream))
    return e.value


def rk3_step_f32(plan, Z, W, phi, nu, dt, stream=None, energy=True):
    e = ctypes.c_double(0.0)
    _call("sph_rk3_step_f32", plan.h, _s32(plan, Z), _s32(plan, W), _s32(plan, phi), float(nu), float(dt),
          ctypes.byref(e) if energy else None, _stream(stream))
    return e.value


# ---------------------------------------------------------------- NL + RK3
def nl_rhs(plan, Z, W, phi, nu, rhs_z, rhs_phi, stream=None):
    e = ctypes.c_double(0.0)
    _call("sph_nl_rhs", plan.h, _s(plan, Z), _s(plan, W), _s(plan, phi), float(nu),
          _s(plan, rhs_z), _s(plan, rhs_phi), ctypes.byref(e), _stream(stream))
    return e.value


def rk3_step(plan, Z, W, phi, nu, dt, stream=None, energy=True):
    e = ctypes.c_double(0.0)
    _call("sph_rk3_step", plan.h, _s(plan, Z), _s(plan, W), _s(plan, phi), float(nu), float(dt),
          ctypes.byref(e) if energy else None, _stream(stream))
    return e.value


# ---------------------------------------------------------------- run loop
def read_namelist(path):
    """&grid, &boxparams and the optional &run group (see sph_read_namelist)."""
    ints = {k: ctypes.c_int() for k in ("lmax", "nz", "Cz", "oz", "step", "tstep", "sstep", "filter")}
    dbls = {k: ctypes.c_double() for k in ("rint", "rext", "dt", "nu")}
    _call("sph_read_namelist", os.fsencode(path), *(ctypes.byref(ints[k]) for k in ("lmax", "nz", "Cz", "oz")),
          ctypes.byref(dbls["rint"]), ctypes.byref(dbls["rext"]), ctypes.byref(dbls["dt"]),
          *(ctypes.byref(ints[k]) for k in ("step", "tstep", "sstep")), ctypes.byref(dbls["nu"]),
          ctypes.byref(ints["filter"]))
    out = {k: v.value for k, v in ints.items()}
    out.update({k: v.value for k, v in dbls.items()})
    out["filter"] = bool(out["filter"])
    return out


def write_grids(plan, dir):
    """theta.txt, phi.txt, z.txt in dir (box_init's grid files)."""
    _call("sph_write_grids", plan.h, os.fsencode(dir))


def energy_spectrum(plan, Z, W, stream=None):
    """Kinetic energy per degree: a list of (toroidal, poloidal) for l = 0..lmax."""
    out = (ctypes.c_double * (2 * (plan.lmax + 1)))()
    _call("sph_energy_spectrum", plan.h, _s(plan, Z), _s(plan, W), out, _stream(stream))
    return [(out[2 * l], out[2 * l + 1]) for l in range(plan.lmax + 1)]


def run(plan, Z, W, phi, nu, dt, nsteps, tstep=1, sstep=0, filter=False, outdir=None, stream=None):
    """nsteps RK3 steps with the optional filter and outputs (see sph_run);
    returns the energy of the final state."""
    e = ctypes.c_double(0.0)
    _call("sph_run", plan.h, _s(plan, Z), _s(plan, W), _s(plan, phi), float(nu), float(dt), int(nsteps),
          int(tstep), int(sstep), int(bool(filter)), os.fsencode(outdir) if outdir else None, ctypes.byref(e),
          _stream(stream))
    return e.value


# ---------------------------------------------------------------- timers
def timer_enable(plan, on=True):
    _call("sph_timer_enable", plan.h, int(bool(on)))


def timer_reset(plan):
    _call("sph_timer_reset", plan.h)


def set_tiles(plan, rows=0, ring_pairs=0, z_cols=0):
    """Tile shapes of the plan's kernels (0: built-in choice); see sph_plan_set_tiles."""
    _call("sph_plan_set_tiles", plan.h, int(rows), int(ring_pairs), int(z_cols))
    plan.tiles = {"rows": int(rows), "ring_pairs": int(ring_pairs), "z_cols": int(z_cols)}


def plan_status(plan):
    """Raises SphError(SPH_ETIMEDOUT) if a bounded device wait of the plan's
    tensor-core kernels gave up since the last check."""
    _call("sph_plan_status", plan.h)


def timer_read(plan):
    """{class: (milliseconds, launches)} accumulated since the last reset."""
    ms = (ctypes.c_double * len(TIMER_CLASSES))()
    n = (ctypes.c_int * len(TIMER_CLASSES))()
    _call("sph_timer_read", plan.h, ms, n)
    return {c: (ms[i], n[i]) for i, c in enumerate(TIMER_CLASSES)}


# ---------------------------------------------------------------- batches
class Batch:
    """Independent problems run together (sph_batch_*): for every field of
    every plan, the inverse 3D transform of `spec` into `grid` (z inverse in
    place), `dspec` = derivr(spec, 1, 'r'), and the forward 3D transform of
    `grid` back into `spec`; one CUDA graph, grouped Legendre launches."""

    def __init__(self, plans, nfields, tuned=True):
        self.plans = list(plans)
        if tuned:  # tile shapes from the autotuner's table, where it has the size
            from redondito_b200 import autotune
            table = autotune.load_table()
            for P in self.plans:
                autotune.apply(P, autotune.tiles_for(P.lmax, P.nz, P.nlat, P.nphi,
                                                     P.precision == SPH_MIXED, table))
        self.nfields = [int(n) for n in nfields]
        self.spec, self.grid, self.dspec = [], [], []
        for P, n in zip(self.plans, self.nfields):
            self.spec.append([P.new_spec() for _ in range(n)])
            self.grid.append([P.new_grid() for _ in range(n)])
            self.dspec.append([P.new_spec() for _ in range(n)])
        flat = [lambda xs=xs: [t for ts in xs for t in ts] for xs in (self.spec, self.grid, self.dspec)]
        arrays = [f() for f in flat]
        ptrs = [(ctypes.c_void_p * len(xs))(*[t.data_ptr() for t in xs]) for xs in arrays]
        ph = (ctypes.c_void_p * len(self.plans))(*[P.h.value for P in self.plans])
        nf = (ctypes.c_int * len(self.nfields))(*self.nfields)
        self._keep = (ph, nf, *ptrs)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.plans[0].device):
            _call("sph_batch_create", ctypes.byref(h), len(self.plans), ph, nf, *ptrs)
        self.h = h

    def run(self, stream=None):
        _call("sph_batch_run", self.h, _stream(stream))

    def status(self):
        _call("sph_batch_status", self.h)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().sph_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
