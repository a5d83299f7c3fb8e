"""ctypes binding of the CPU oracle (oracle/sph_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline / reference arm.  The product never imports it.

Arrays follow the reference layouts (see sph_oracle.h):
  grid  float64 (nz, nphi, nlat)   -- Fortran REAL (nlat,nphi,nz)
  spec  complex128 (nz, nlm)       -- Fortran COMPLEX (nlm,nz)
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsph_oracle.so")
TABLES_DIR = os.path.join(os.path.dirname(_HERE), "redondito_b200", "tables")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "sph_oracle.cpp")
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        I = ctypes.c_int
        L.orc_plan_create.restype = P
        L.orc_plan_create.argtypes = [I, I, I, I, I, I, ctypes.c_double, ctypes.c_double, D]
        L.orc_plan_destroy.argtypes = [P]
        L.orc_nlm.argtypes = [P]
        L.orc_set_threads.argtypes = [I]
        L.orc_load_dirichlet_tables.argtypes = [ctypes.c_char_p, I, I, D]
        L.orc_grid.argtypes = [P, D, D, D, D, D, ctypes.POINTER(I), ctypes.POINTER(I)]
        for name in ("orc_sh_analysis", "orc_sh_synthesis", "orc_3d_forward", "orc_3d_inverse",
                     "orc_laplang", "orc_dlr", "orc_copy", "orc_invDl"):
            getattr(L, name).argtypes = [P, D, D]
        for name in ("orc_z_forward", "orc_z_inverse", "orc_dirichlet"):
            getattr(L, name).argtypes = [P, D]
        L.orc_z_forward_cols.argtypes = [P, D, I]
        L.orc_z_inverse_cols.argtypes = [P, D, I]
        L.orc_qst_analysis.argtypes = [P] + [D] * 6
        L.orc_qst_synthesis.argtypes = [P] + [D] * 6
        L.orc_derivr.argtypes = [P, D, D, I, ctypes.c_char]
        L.orc_multr.argtypes = [P, D, D, I]
        L.orc_saxpby_c.argtypes = [P, D, D, ctypes.c_double, D, ctypes.c_double]
        L.orc_saxpby_r.argtypes = [P, D, D, ctypes.c_double, D, ctypes.c_double]
        L.orc_fc_filter.argtypes = [P, D, ctypes.c_char]
        L.orc_prodvec.argtypes = [P] + [D] * 9
        L.orc_bc_setup.argtypes = [P]
        L.orc_derivr_mat.argtypes = [P, I, D]
        L.orc_imposebc.argtypes = [P, D, D, D, I]
        L.orc_bc_tables.argtypes = [P, D, D]
        L.orc_nl_rhs.argtypes = [P, D, D, D, ctypes.c_double, D, D, D]
        L.orc_rk3_step.argtypes = [P, D, D, D, ctypes.c_double, ctypes.c_double, D]
        L.orc_velocity.argtypes = [P] + [D] * 9
        L.orc_energy_spectrum.argtypes = [P, D, D, D]
        L.orc_load_neumann_tables.argtypes = [ctypes.c_char_p, I, I, ctypes.c_double, D]
        L.orc_set_neumann.argtypes = [P, D, D]
        L.orc_set_neumann.restype = None
        L.orc_neumann_reconstruct.argtypes = [P, D, I, I]
        L.orc_robin_reconstruct.argtypes = [P, D, I, D]
        L.orc_bc_setup_kinds.argtypes = [P, I, I]
        L.orc_bc_set_tables.argtypes = [P, I, I, D, D]
        for name in ("orc_plan_destroy", "orc_set_threads", "orc_grid", "orc_sh_analysis",
                     "orc_sh_synthesis", "orc_qst_analysis", "orc_qst_synthesis", "orc_z_forward",
                     "orc_z_inverse", "orc_3d_forward", "orc_3d_inverse", "orc_laplang",
                     "orc_multr", "orc_dlr", "orc_saxpby_c", "orc_saxpby_r", "orc_copy",
                     "orc_prodvec", "orc_dirichlet", "orc_derivr_mat", "orc_invDl",
                     "orc_imposebc", "orc_bc_tables", "orc_nl_rhs", "orc_rk3_step",
                     "orc_velocity", "orc_z_forward_cols", "orc_z_inverse_cols",
                     "orc_energy_spectrum"):
            getattr(L, name).restype = None
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n):
    lib().orc_set_threads(int(n))


def load_dir(C=25, d=5, tdir=TABLES_DIR):
    out = np.zeros(C * d)
    rc = lib().orc_load_dirichlet_tables(tdir.encode(), C, d, _p(out))
    if rc:
        raise FileNotFoundError(f"FC-Gram tables A{C}-{d}.dat/Q{d}.dat not readable in {tdir}")
    return out


def load_neumann(d=5, ord=1, dx=1.0, tdir=TABLES_DIR):
    out = np.zeros(d)
    rc = lib().orc_load_neumann_tables(tdir.encode(), d, ord, float(dx), _p(out))
    if rc:
        raise FileNotFoundError(f"Neumann tables Q{d}.dat/Q{ord}n{d}.dat not readable in {tdir} ({rc})")
    return out


def nlat_for(lmax):
    """grid_init rule (pseudospec_mod.f90:67): nlat = 4*((3(lmax+1)+7)/8)."""
    return 4 * ((3 * (lmax + 1) + 7) // 8)


class Plan:
    """Oracle plan: grid + FC-Gram continuation + (optionally) boundary tables."""

    def __init__(self, lmax, nz, nlat=None, nphi=None, C=0, d=0, rint=0.35, rext=1.0, dir=None):
        self.lmax = lmax
        self.nlat = nlat if nlat is not None else nlat_for(lmax)
        self.nphi = nphi if nphi is not None else 2 * self.nlat
        self.nz, self.C, self.d = nz, C, d
        self.rint, self.rext = rint, rext
        if C > 0 and dir is None:
            dir = load_dir(C, d)
        self.dir = None if dir is None else np.ascontiguousarray(dir, dtype=np.float64)
        self.h = lib().orc_plan_create(lmax, self.nlat, self.nphi, nz, C, d, rint, rext,
                                       _p(self.dir))
        if not self.h:
            raise ValueError("orc_plan_create rejected the sizes")
        self.nlm = (lmax + 1) * (lmax + 2) // 2
        self.N = nz - C
        self.theta = np.zeros(self.nlat)
        self.ct = np.zeros(self.nlat)
        self.w = np.zeros(self.nlat)
        self.z = np.zeros(nz)
        self.kz = np.zeros(nz)
        self.ell = np.zeros(self.nlm, dtype=np.int32)
        self.emm = np.zeros(self.nlm, dtype=np.int32)
        lib().orc_grid(self.h, _p(self.theta), _p(self.ct), _p(self.w), _p(self.z), _p(self.kz),
                       self.ell.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                       self.emm.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        self.phi = 2 * np.pi * np.arange(self.nphi) / self.nphi
        self._bc = False
        self.dz = (rext - rint) / (nz - C - 1) if nz - C > 1 else 1.0
        self.neu = None
        if C > 0 and os.path.exists(os.path.join(TABLES_DIR, f"Q1n{d}.dat")):
            self.neu = (load_neumann(d, 1, self.dz), load_neumann(d, 2, self.dz))
            lib().orc_set_neumann(self.h, _p(self.neu[0]), _p(self.neu[1]))

    def __del__(self):
        try:
            if self.h:
                lib().orc_plan_destroy(self.h)
        except Exception:
            pass

    # helpers
    def lm(self, l, m):
        return m * (2 * self.lmax + 1 - m) // 2 + l

    def grid_shape(self):
        return (self.nz, self.nphi, self.nlat)

    def spec_shape(self):
        return (self.nz, self.nlm)

    def new_grid(self):
        return np.zeros(self.grid_shape())

    def new_spec(self):
        return np.zeros(self.spec_shape(), dtype=np.complex128)

    def angles(self):
        """cos(theta), sin(theta), phi broadcast to a (nphi, nlat) plane."""
        cth = np.broadcast_to(self.ct[None, :], (self.nphi, self.nlat))
        sth = np.broadcast_to(np.sin(self.theta)[None, :], (self.nphi, self.nlat))
        ph = np.broadcast_to(self.phi[:, None], (self.nphi, self.nlat))
        return cth, sth, ph

    # transforms (inputs preserved, outputs returned)
    def sh_analysis(self, grid):
        g = np.ascontiguousarray(grid, dtype=np.float64)
        out = self.new_spec()
        lib().orc_sh_analysis(self.h, _p(g), _p(out.view(np.float64)))
        return out

    def sh_synthesis(self, spec):
        s = np.ascontiguousarray(spec, dtype=np.complex128)
        out = self.new_grid()
        lib().orc_sh_synthesis(self.h, _p(s.view(np.float64)), _p(out))
        return out

    def qst_analysis(self, vr, vt, vp):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (vr, vt, vp)]
        q, s, t = self.new_spec(), self.new_spec(), self.new_spec()
        lib().orc_qst_analysis(self.h, *[_p(x) for x in a],
                               *[_p(x.view(np.float64)) for x in (q, s, t)])
        return q, s, t

    def qst_synthesis(self, q, s, t):
        a = [np.ascontiguousarray(x, dtype=np.complex128) for x in (q, s, t)]
        out = [self.new_grid() for _ in range(3)]
        lib().orc_qst_synthesis(self.h, *[_p(x.view(np.float64)) for x in a], *[_p(x) for x in out])
        return tuple(out)

    def z_forward(self, spec):
        s = np.array(spec, dtype=np.complex128, order="C", copy=True)
        lib().orc_z_forward(self.h, _p(s.view(np.float64)))
        return s

    def z_inverse(self, spec):
        s = np.array(spec, dtype=np.complex128, order="C", copy=True)
        lib().orc_z_inverse(self.h, _p(s.view(np.float64)))
        return s

    def z_forward_cols(self, spec):
        """z forward of a (nz, ncols) slice of lm columns (in place on a copy)."""
        s = np.array(spec, dtype=np.complex128, order="C", copy=True)
        assert s.shape[0] == self.nz
        lib().orc_z_forward_cols(self.h, _p(s.view(np.float64)), s.shape[1])
        return s

    def z_inverse_cols(self, spec):
        s = np.array(spec, dtype=np.complex128, order="C", copy=True)
        assert s.shape[0] == self.nz
        lib().orc_z_inverse_cols(self.h, _p(s.view(np.float64)), s.shape[1])
        return s

    def forward_3d(self, grid):
        g = np.ascontiguousarray(grid, dtype=np.float64)
        out = self.new_spec()
        lib().orc_3d_forward(self.h, _p(g), _p(out.view(np.float64)))
        return out

    def inverse_3d(self, spec):
        s = np.ascontiguousarray(spec, dtype=np.complex128)
        out = self.new_grid()
        lib().orc_3d_inverse(self.h, _p(s.view(np.float64)), _p(out))
        return out

    def _un(self, name, a, *extra):
        x = np.ascontiguousarray(a, dtype=np.complex128)
        out = self.new_spec()
        rc = getattr(lib(), name)(self.h, _p(x.view(np.float64)), _p(out.view(np.float64)), *extra)
        if rc not in (None, 0):
            raise ValueError(f"{name} failed ({rc})")
        return out

    def derivr(self, a, order, esp="r"):
        return self._un("orc_derivr", a, order, esp.encode())

    def laplang(self, a):
        return self._un("orc_laplang", a)

    def multr(self, a, power):
        return self._un("orc_multr", a, power)

    def dlr(self, a):
        return self._un("orc_dlr", a)

    def copy(self, a):
        return self._un("orc_copy", a)

    def saxpby_c(self, x, a, y, b):
        xx = np.ascontiguousarray(x, dtype=np.complex128)
        yy = np.ascontiguousarray(y, dtype=np.complex128)
        out = self.new_spec()
        lib().orc_saxpby_c(self.h, _p(out.view(np.float64)), _p(xx.view(np.float64)), a,
                           _p(yy.view(np.float64)), b)
        return out

    def saxpby_r(self, x, a, y, b):
        xx = np.ascontiguousarray(x, dtype=np.float64)
        yy = np.ascontiguousarray(y, dtype=np.float64)
        out = self.new_grid()
        lib().orc_saxpby_r(self.h, _p(out), _p(xx), a, _p(yy), b)
        return out

    def fc_filter(self, a, esp="r"):
        s = np.array(a, dtype=np.complex128, order="C", copy=True)
        rc = lib().orc_fc_filter(self.h, _p(s.view(np.float64)), esp.encode())
        if rc:
            raise ValueError("fc_filter failed")
        return s

    def prodvec(self, A, B):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (*A, *B)]
        out = [self.new_grid() for _ in range(3)]
        lib().orc_prodvec(self.h, *[_p(x) for x in a], *[_p(x) for x in out])
        return tuple(out)

    def dirichlet(self, a):
        s = np.array(a, dtype=np.complex128, order="C", copy=True)
        lib().orc_dirichlet(self.h, _p(s.view(np.float64)))
        return s

    def bc_setup(self, kinds=None, tables=None):
        """Boundary kinds at the inner and outer wall: noslip or freeslip
        (None: keep the kinds set up, noslip if none).  tables = (binv,
        d2bor) in bc_tables()'s layouts replaces the matrices invDl_setup
        builds (e.g. extended.bc_tables(), evaluated in long double)."""
        code = {"noslip": 0, "freeslip": 1}
        if kinds is None:
            if self._bc:
                return
            kinds = ("noslip", "noslip")
        k = (code[kinds[0]], code[kinds[1]])
        if tables is not None:
            binv = np.ascontiguousarray(tables[0], dtype=np.float64).ravel()
            d2bor = np.ascontiguousarray(tables[1], dtype=np.float64).ravel()
            assert binv.size == self.N * (self.N - 4) * max(self.lmax, 1) and d2bor.size == 4 * self.N
            rc = lib().orc_bc_set_tables(self.h, *k, _p(binv), _p(d2bor))
            if rc:
                raise ValueError(f"bc_set_tables failed ({rc})")
            self._bc = True
            self._bck = k
            return
        if not self._bc or getattr(self, "_bck", (0, 0)) != k:
            rc = lib().orc_bc_setup_kinds(self.h, *k)
            if rc:
                raise ValueError(f"bc_setup failed ({rc})")
            self._bc = True
            self._bck = k

    def neumann_reconstruct(self, a, boun, ord=1):
        """The boundary row (boun 0 inner, 1 outer) of a copy of a, from the
        ord-th outward normal derivative held there."""
        s = np.array(a, dtype=np.complex128, order="C", copy=True)
        if lib().orc_neumann_reconstruct(self.h, _p(s.view(np.float64)), boun, ord):
            raise ValueError("neumann_reconstruct failed")
        return s

    def robin_reconstruct(self, a, boun, coef):
        s = np.array(a, dtype=np.complex128, order="C", copy=True)
        c = np.ascontiguousarray(np.broadcast_to(np.asarray(coef, dtype=np.float64), (self.nlm,)))
        if lib().orc_robin_reconstruct(self.h, _p(s.view(np.float64)), boun, _p(c)):
            raise ValueError("robin_reconstruct failed")
        return s

    def derivr_mat(self, order):
        d = np.zeros((self.N, self.N), order="F")
        buf = np.zeros(self.N * self.N)
        lib().orc_derivr_mat(self.h, order, _p(buf))
        return buf.reshape(self.N, self.N, order="F")

    def bc_tables(self):
        self.bc_setup()
        n = self.N
        binv = np.zeros(n * (n - 4) * max(self.lmax, 1))
        d2bor = np.zeros(4 * n)
        lib().orc_bc_tables(self.h, _p(binv), _p(d2bor))
        return binv.reshape(max(self.lmax, 1), n - 4, n), d2bor.reshape(n, 4)

    def invDl(self, phi):
        self.bc_setup()
        return self._un("orc_invDl", phi)

    def imposebc(self, tor, phi, fast=False):
        self.bc_setup()
        t = np.array(tor, dtype=np.complex128, order="C", copy=True)
        f = np.array(phi, dtype=np.complex128, order="C", copy=True)
        w = self.new_spec()
        lib().orc_imposebc(self.h, _p(t.view(np.float64)), _p(f.view(np.float64)),
                           _p(w.view(np.float64)), int(fast))
        return t, f, w

    def nl_rhs(self, Z, W, phi, nu):
        self.bc_setup()
        a = [np.ascontiguousarray(x, dtype=np.complex128) for x in (Z, W, phi)]
        rz, rf = self.new_spec(), self.new_spec()
        e = np.zeros(1)
        lib().orc_nl_rhs(self.h, *[_p(x.view(np.float64)) for x in a], nu,
                         _p(rz.view(np.float64)), _p(rf.view(np.float64)), _p(e))
        return rz, rf, float(e[0])

    def rk3_step(self, Z, W, phi, nu, dt):
        self.bc_setup()
        a = [np.array(x, dtype=np.complex128, order="C", copy=True) for x in (Z, W, phi)]
        e = np.zeros(1)
        lib().orc_rk3_step(self.h, *[_p(x.view(np.float64)) for x in a], nu, dt, _p(e))
        return a[0], a[1], a[2], float(e[0])

    def energy_spectrum(self, Z, W):
        """(lmax+1, 2): toroidal and poloidal kinetic energy per degree l."""
        a = [np.ascontiguousarray(x, dtype=np.complex128) for x in (Z, W)]
        out = np.zeros(2 * (self.lmax + 1))
        lib().orc_energy_spectrum(self.h, *[_p(x.view(np.float64)) for x in a], _p(out))
        return out.reshape(self.lmax + 1, 2)

    def velocity(self, Z, W, phi, vorticity=True):
        a = [np.ascontiguousarray(x, dtype=np.complex128) for x in (Z, W, phi)]
        out = [self.new_grid() for _ in range(6 if vorticity else 3)]
        ptrs = [_p(x) for x in out] + ([None] * 3 if not vorticity else [])
        lib().orc_velocity(self.h, *[_p(x.view(np.float64)) for x in a], *ptrs)
        return tuple(out)
