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


def test_range_matches_the_reference_rule():
    """sph_range against range (src/sphp/sphp_sca.F90:596-626) restated here:
    the parts tile [n1, n2] in order, sizes differ by at most one, the
    first mod(n, nprocs) ranks take the extra element."""
    from redondito_b200 import sphp as S
    for n1, n2 in ((1, 1), (1, 7), (0, 63), (1, 131328), (5, 4)):
        for nprocs in range(1, 7):
            parts = [S.range_(n1, n2, nprocs, r) for r in range(nprocs)]
            n = n2 - n1 + 1
            w1, w2 = divmod(n, nprocs)
            for r, (a, b) in enumerate(parts):
                ista = r * w1 + n1 + min(r, w2)
                iend = ista + w1 - 1 + (1 if w2 > r else 0)
                assert (a, b) == (ista, iend)
            assert parts[0][0] == n1 and parts[-1][1] == n2
            for (a0, b0), (a1, b1) in zip(parts, parts[1:]):
                assert a1 == b0 + 1
