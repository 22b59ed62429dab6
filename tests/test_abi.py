"""CPU tests of the boundary: the C-ABI library loads and exports every symbol the header declares."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include"))) if f.endswith(".h")]


def declared():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:int|const char\*|void)\s+(mpm_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from physbam_b200 import build
    build.build()
    return ctypes.CDLL(build.LIB)


def test_header_declares_entry_points():
    names = declared()
    for must in ("mpm_create", "mpm_destroy", "mpm_set_particles", "mpm_get_particles", "mpm_substep",
                 "mpm_advance", "mpm_set_collision_objects", "mpm_get_grid", "mpm_radix_sort_u32"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(lib):
    lib.mpm_status_string.restype = ctypes.c_char_p
    assert lib.mpm_status_string(0) == b"ok"
    assert lib.mpm_status_string(4) == b"particle outside the grid"


def test_argument_checks_need_no_gpu(lib):
    """Bad descriptors are rejected before any CUDA call."""
    from physbam_b200 import driver as D
    g = D.GridDesc()
    g.dim = 4
    m = D.ModelDesc()
    h = ctypes.c_void_p()
    assert lib.mpm_create(ctypes.byref(g), ctypes.byref(m), ctypes.byref(h)) == 1
    g.dim, g.ghost = 3, 2
    assert lib.mpm_create(ctypes.byref(g), ctypes.byref(m), ctypes.byref(h)) == 1
    g.ghost = 3
    g.counts[0] = g.counts[1] = g.counts[2] = 16
    for a in range(3):
        g.domain_max[a] = 1.0
    m.path, m.precision = 0, 1    # the fast path is FP32 only
    assert lib.mpm_create(ctypes.byref(g), ctypes.byref(m), ctypes.byref(h)) == 1
    k = np.zeros(4, np.uint32)
    assert lib.mpm_radix_sort_u32(ctypes.c_void_p(k.ctypes.data), ctypes.c_int64(4), 0,
                                  ctypes.c_void_p(k.ctypes.data), ctypes.c_void_p(k.ctypes.data)) == 1


def test_driver_refuses_without_library(tmp_path):
    from physbam_b200 import driver as D
    saved = D._lib
    D._lib = None
    try:
        with pytest.raises(RuntimeError, match="no CPU fallback"):
            D.load_library(str(tmp_path / "missing.so"))
    finally:
        D._lib = saved
