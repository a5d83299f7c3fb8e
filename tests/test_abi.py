"""The C-ABI library builds for sm_100a, loads without a GPU and exports
every function include/sph_b200.h declares (no compute calls here)."""
import os
import re

from redondito_b200 import build as B


def declared_symbols():
    hdr = open(os.path.join(B.ROOT, "include", "sph_b200.h")).read()
    return sorted(set(re.findall(r"\bint\s+(sph_\w+)\s*\(", hdr)))


def test_library_exports_header(tmp_path):
    import ctypes
    lib = ctypes.CDLL(B.build())
    names = declared_symbols()
    assert len(names) >= 29
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_covers_header():
    from redondito_b200 import sphp as S
    assert sorted(S.SYMBOLS) == declared_symbols()


def test_invalid_sizes_rejected_without_gpu():
    # argument checks run before any CUDA call
    import ctypes
    from redondito_b200 import sphp as S
    L = S.lib()
    h = ctypes.c_void_p()
    assert L.sph_plan_create(ctypes.byref(h), 31, 47, 96, 33, 0, 0, 0.35, 1.0, None, 0) == 1  # odd nlat
    assert L.sph_plan_create(ctypes.byref(h), 31, 48, 62, 33, 0, 0, 0.35, 1.0, None, 0) == 1  # nphi <= 2 lmax
    assert L.sph_plan_create(ctypes.byref(h), 31, 48, 96, 33, 25, 5, 0.35, 1.0, None, 0) == 1  # no dir table
    assert L.sph_setup_bc(None, b"noslip", b"noslip") == 1
    d = (ctypes.c_double * 125)()
    assert L.sph_fcgram_load_tables(b"/nonexistent", 25, 5, d) == 5


def test_fcgram_tables_match_generator_definition():
    import ctypes
    import numpy as np
    from redondito_b200 import sphp as S
    d = np.array(S.load_dirichlet_tables(25, 5)).reshape(5, 25).T
    A = np.fromfile(os.path.join(S.TABLES_DIR, "A25-5.dat")).reshape(5, 25).T
    Q = np.fromfile(os.path.join(S.TABLES_DIR, "Q5.dat")).reshape(5, 5).T
    assert np.abs(d - A @ Q.T).max() < 1e-12
