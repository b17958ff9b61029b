"""C ABI checks that need no GPU: the library loads, exports every function
include/fwi2d_b200.h declares, computes the reference's injector tables on the
host, and reports errors as status codes."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import fwi2d_b200 as F
from fwi2d_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def header_functions():
    txt = open(os.path.join(ROOT, "include", "fwi2d_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fwi2d_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    L = F.load()
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) <= set(C.SYMBOLS)


def test_injector_weights_match_reference_tables():
    files = sorted(glob.glob(os.path.join(GOLD, "*_f32.npz")))
    n = 0
    for f in files:
        g = dict(np.load(f))
        if "src_xind" not in g:
            continue
        nx, nz, d = int(g["nx"]), int(g["nz"]), float(g["d"])
        mt = int(g["mt"])
        t = F.injector_tables(1 if mt else 0, g["src_x"], g["src_z"], nx, nz, d, d, 0.0, 0.0)
        for a, b in zip(t, (g["src_xind"], g["src_zind"], g["src_xw"], g["src_zw"])):
            assert np.array_equal(a, b), f
        t = F.injector_tables(0, g["rcv_x"], g["rcv_z"], nx, nz, d, d, 0.0, 0.0)
        for a, b in zip(t, (g["rcv_xind"], g["rcv_zind"], g["rcv_xw"], g["rcv_zw"])):
            assert np.array_equal(a, b), f
        n += 1
    assert n >= 5


def test_boundary_pivots_shift_inward():
    """delta_m3 moves a pivot on the first or last sample one cell inward
    (injector.cpp:31-37)."""
    xind, zind, xw, zw = F.injector_tables(0, [0.0, 0.59], [0.0, 0.39], 60, 40, 0.01, 0.01, 0.0, 0.0)
    assert list(xind[0]) == [0, 1, 2] and list(zind[0]) == [0, 1, 2]
    assert list(xind[1]) == [57, 58, 59] and list(zind[1]) == [37, 38, 39]


def test_errors_are_status_codes():
    L = F.load()
    rc = L.fwi2d_injector_weights(7, 1, None, None, 10, 10, 1.0, 1.0, 0.0, 0.0, None, None, None, None)
    assert rc == -1 and b"injector" in L.fwi2d_last_error()
    h = ctypes.c_void_p()
    rc = L.fwi2d_ctx_create(-1, ctypes.byref(h))
    assert rc != 0 and len(L.fwi2d_last_error()) > 0
    shape = (ctypes.c_int(), ctypes.c_int())
    assert L.fwi2d_tile_shape(0, ctypes.byref(shape[0]), ctypes.byref(shape[1])) == 0
    assert shape[0].value % 32 == 0 and shape[1].value >= 8
    assert L.fwi2d_tile_shape(99, ctypes.byref(shape[0]), ctypes.byref(shape[1])) == -1
