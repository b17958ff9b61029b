"""fwi2d_propagate_noalloc: the allocation-free forward entry point.

It serves callers that cannot allocate device memory: plug-ins whose host
framework owns the device allocator and must account for every byte, and
real-time loops that may not call the device-synchronising cudaMalloc /
cudaFree once they run.  All its device buffers live in one static array
inside the library.

The checks:
* two calls in a row through the C ABI each reproduce the regular
  fwi2d_propagate forward (same tolerance as the other parity tests; in
  practice bitwise), over several boundary-condition sets, a top taper and a
  receiver buffer that already holds data (the entry point accumulates into
  it), so the shared array leaves nothing behind from the previous call;
* as the first library call of a fresh process it sets up the device itself
  and gives the same receivers;
* after a first call has reserved the array, a further call leaves the
  device's free memory unchanged: it allocates nothing;
* incomplete injector tables and problems larger than the array are
  rejected with an error code.
Collected last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process.
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


def _case(seed, nx, nz, nt, nr, bc=(1, 2, 2, 2), taper=(0, 8, 8, 8)):
    d = 0.01
    mc = K.converted(0, K.model_case(0, nx, nz, d, seed=seed))
    sl, rl = K.geometry(nx, nz, d, nr=nr)
    src = np.ascontiguousarray(K.sources(2, nt, 1e-3))
    inj = F.injector_tables(0, sl[0], sl[1], nx, nz, d, d, 0, 0)
    ext = F.injector_tables(0, rl[0], rl[1], nx, nz, d, d, 0, 0)
    params = F.make_params(**K.par_dict(nt=nt, dt=1e-3, sub=0, bc=bc, taper=taper))
    return mc, src, inj, ext, params, d


def _injector(t):
    return C.Injector(0, len(t[0]), C.ptr(t[0]), C.ptr(t[1]), C.ptr(t[2]), C.ptr(t[3]))


def _noalloc(L, mc, src, out, ji, je, params, nr, nx, nz, d):
    return L.fwi2d_propagate_noalloc(C.ptr(mc), C.ptr(src), C.ptr(out), ctypes.byref(ji), ctypes.byref(je),
                                     ctypes.byref(params), 1, nr, nx, nz, d, d)


CASES = [
    # seed, nx, nz, nt, nr, bc (top, bottom, left, right), taper (top, bottom, left, right)
    (7, 96, 80, 160, 20, (1, 2, 2, 2), (0, 8, 8, 8)),
    (8, 72, 104, 140, 16, (1, 2, 2, 2), (0, 8, 8, 8)),
    (9, 80, 72, 150, 12, (2, 2, 2, 2), (6, 8, 8, 8)),
    (10, 88, 76, 130, 14, (2, 1, 1, 2), (5, 0, 7, 9)),
]


@pytest.mark.parametrize("seed,nx,nz,nt,nr,bc,taper", CASES)
def test_noalloc_matches_propagate_twice(seed, nx, nz, nt, nr, bc, taper):
    L = _bind(F.load())
    mc, src, inj, ext, params, d = _case(seed, nx, nz, nt, nr, bc, taper)
    ji, je = _injector(inj), _injector(ext)
    # receivers are accumulated into what the buffer already holds
    base = np.random.default_rng(seed).standard_normal((2, nr, nt)).astype(np.float32)
    ref = base.copy()
    C.check(L.fwi2d_propagate(0, 0, C.ptr(mc), C.ptr(src), C.ptr(ref), ctypes.byref(ji), ctypes.byref(je),
                              None, None, None, None, ctypes.byref(params), 1, nr, nx, nz, d, d))
    for call in range(2):
        out = base.copy()
        rc = _noalloc(L, mc, src, out, ji, je, params, nr, nx, nz, d)
        assert rc == 0, L.fwi2d_noalloc_last_error().decode()
        err = K.rel_l2(out - base, ref - base)
        assert err <= TRACE_TOL, "call %d: rel-L2 %.3e" % (call, err)


FRESH = r'''
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import fwi2d_b200 as F
from fwi2d_b200 import _capi as C
from tests import test_zz_no_alloc as T
L = T._bind(F.load())
seed, nx, nz, nt, nr, bc, taper = T.CASES[0]
mc, src, inj, ext, params, d = T._case(seed, nx, nz, nt, nr, bc, taper)
out = np.zeros((2, nr, nt), np.float32)
rc = T._noalloc(L, mc, src, out, T._injector(inj), T._injector(ext), params, nr, nx, nz, d)
assert rc == 0, L.fwi2d_noalloc_last_error().decode()
np.save(sys.argv[2], out)
'''


def test_noalloc_first_call_in_fresh_process(tmp_path):
    """The entry point is the first library call of a fresh process (no
    context was ever created there): it must set up the device itself."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    path = str(tmp_path / "rcv.npy")
    subprocess.run([sys.executable, "-c", FRESH, root, path], check=True, timeout=600)
    out = np.load(path)
    L = _bind(F.load())
    seed, nx, nz, nt, nr, bc, taper = CASES[0]
    mc, src, inj, ext, params, d = _case(seed, nx, nz, nt, nr, bc, taper)
    ref = np.zeros((2, nr, nt), np.float32)
    C.check(L.fwi2d_propagate(0, 0, C.ptr(mc), C.ptr(src), C.ptr(ref), ctypes.byref(_injector(inj)),
                              ctypes.byref(_injector(ext)), None, None, None, None, ctypes.byref(params), 1, nr, nx, nz,
                              d, d))
    assert K.rel_l2(out, ref) <= TRACE_TOL


def test_noalloc_call_allocates_no_device_memory():
    import torch
    L = _bind(F.load())
    seed, nx, nz, nt, nr, bc, taper = CASES[0]
    mc, src, inj, ext, params, d = _case(seed, nx, nz, nt, nr, bc, taper)
    ji, je = _injector(inj), _injector(ext)
    out = np.zeros((2, nr, nt), np.float32)
    # the first call on the device reserves the static array (lazy module loading)
    assert _noalloc(L, mc, src, out, ji, je, params, nr, nx, nz, d) == 0, L.fwi2d_noalloc_last_error().decode()
    torch.cuda.synchronize(0)
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(2):
        out[:] = 0
        assert _noalloc(L, mc, src, out, ji, je, params, nr, nx, nz, d) == 0, L.fwi2d_noalloc_last_error().decode()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, "device free memory changed by %d bytes" % (free0 - free1)


def test_noalloc_rejects_incomplete_tables():
    L = _bind(F.load())
    seed, nx, nz, nt, nr, bc, taper = CASES[0]
    mc, src, inj, ext, params, d = _case(seed, nx, nz, nt, nr, bc, taper)
    ji, je = _injector(inj), _injector(ext)
    out = np.zeros((2, nr, nt), np.float32)
    for field in ("xind", "zind", "xw", "zw"):
        for J in (ji, je):
            keep = getattr(J, field)
            setattr(J, field, None)
            rc = _noalloc(L, mc, src, out, ji, je, params, nr, nx, nz, d)
            setattr(J, field, keep)
            assert rc == -1
            assert b"incomplete" in L.fwi2d_noalloc_last_error()


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
