"""fwi2d_propagate_noalloc: the allocation-free forward entry point.

It serves callers that cannot allocate device memory (plug-ins whose host
framework owns the device allocator, real-time loops that may not call the
device-synchronising cudaMalloc / cudaFree); all its device buffers live in
one static array inside the library.
The check: two calls in a row through the C ABI each reproduce the regular
fwi2d_propagate forward (same tolerance as the other parity tests; in
practice bitwise), so the shared scratch leaves nothing behind from the
previous call.  Collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import fwi2d_b200 as F
from fwi2d_b200 import _capi as C
from tests import cases as K

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-6


def _bind(L):
    vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.fwi2d_propagate_noalloc.argtypes = [vp, vp, vp, vp, vp, ctypes.POINTER(C.Params), i, i, i, i, f, f]
    L.fwi2d_noalloc_last_error.restype = ctypes.c_char_p
    return L


def _case(seed, nx, nz, nt, nr):
    d = 0.01
    mc = K.converted(0, K.model_case(0, nx, nz, d, seed=seed))
    sl, rl = K.geometry(nx, nz, d, nr=nr)
    src = np.ascontiguousarray(K.sources(2, nt, 1e-3))
    inj = F.injector_tables(0, sl[0], sl[1], nx, nz, d, d, 0, 0)
    ext = F.injector_tables(0, rl[0], rl[1], nx, nz, d, d, 0, 0)
    params = F.make_params(**K.par_dict(nt=nt, dt=1e-3, sub=0))
    return mc, src, inj, ext, params, d


def _injector(t):
    return C.Injector(0, len(t[0]), C.ptr(t[0]), C.ptr(t[1]), C.ptr(t[2]), C.ptr(t[3]))


def test_noalloc_matches_propagate_twice():
    L = _bind(F.load())
    for seed, nx, nz, nt, nr in [(7, 96, 80, 160, 20), (8, 72, 104, 140, 16)]:
        mc, src, inj, ext, params, d = _case(seed, nx, nz, nt, nr)
        ji, je = _injector(inj), _injector(ext)
        ref = np.zeros((2, nr, nt), np.float32)
        C.check(L.fwi2d_propagate(0, 0, C.ptr(mc), C.ptr(src), C.ptr(ref), ctypes.byref(ji), ctypes.byref(je),
                                  None, None, None, None, ctypes.byref(params), 1, nr, nx, nz, d, d))
        for call in range(2):
            out = np.zeros((2, nr, nt), np.float32)
            rc = L.fwi2d_propagate_noalloc(C.ptr(mc), C.ptr(src), C.ptr(out), ctypes.byref(ji), ctypes.byref(je),
                                           ctypes.byref(params), 1, nr, nx, nz, d, d)
            assert rc == 0, L.fwi2d_noalloc_last_error().decode()
            err = K.rel_l2(out, ref)
            assert err <= TRACE_TOL, "call %d: rel-L2 %.3e" % (call, err)


def test_noalloc_rejects_oversized_problem():
    L = _bind(F.load())
    nx, nz, nt, nr = 64, 64, 20000, 1000      # 160 MB of receiver traces: more than the static scratch
    mc = np.ones((3, nx, nz), np.float32)
    tiny = np.zeros(4, np.float32)            # never read: the size check comes first
    inj = F.injector_tables(0, [0.3], [0.1], nx, nz, 0.01, 0.01, 0, 0)
    ext = F.injector_tables(0, np.full(nr, 0.3, np.float32), np.full(nr, 0.1, np.float32), nx, nz, 0.01, 0.01, 0, 0)
    params = F.make_params(**K.par_dict(nt=nt, dt=1e-3, sub=0))
    rc = L.fwi2d_propagate_noalloc(C.ptr(mc), C.ptr(tiny), C.ptr(tiny), ctypes.byref(_injector(inj)),
                                   ctypes.byref(_injector(ext)), ctypes.byref(params), 1, nr, nx, nz, 0.01, 0.01)
    assert rc == -1
    assert b"scratch" in L.fwi2d_noalloc_last_error()
