"""Dipole (distributed acoustic sensing) receivers through the propagate_gpu
drop-in: fwi2d_propagate with a dipole_m3 injector (src/cpp/injector.cpp:
241-380) as the receivers of the forward and the injector of the adjoint, on
the elastic propagator, against the reference's own outputs
(tests/golden/dipole_f32.npz, written by its build).

The library extracts each end as a delta receiver and subtracts, where the
reference sums the nine per-cell differences; the products are the same and
only the summation order differs, so the bars are relative L2 1e-6 for the
traces and 1e-5 for the gradient rather than bit equality.
"""
import ctypes
import os

import numpy as np
import pytest

import fwi2d_b200 as F
from fwi2d_b200 import _capi as C
from fwi2d_b200.propagator import dipole_tables
from tests import cases as K

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_dropin_dipole_receivers_match_reference():
    g = dict(np.load(os.path.join(GOLD, "dipole_f32.npz")))
    kind, nx, nz, d, nt = int(g["kind"]), int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nt"])
    nr = len(g["rx"])
    L = F.load()
    inj = F.injector_tables(0, [float(g["sx"])], [float(g["sz"])], nx, nz, d, d, 0, 0)
    dip = dipole_tables(g["rx"], g["rz"], g["rdip"], float(g["gl"]), nx, nz, d, d)
    ji = C.Injector(C.INJ_DELTA, 1, C.ptr(inj[0]), C.ptr(inj[1]), C.ptr(inj[2]), C.ptr(inj[3]))
    jd = C.Injector(C.INJ_DIPOLE, nr, C.ptr(dip[0]), C.ptr(dip[1]), C.ptr(dip[2]), C.ptr(dip[3]))
    params = F.make_params(**K.par_dict(nt=nt, dt=1e-3))
    mc = np.ascontiguousarray(g["model"])
    rcv = np.zeros((2, nr, nt), np.float32)
    full = np.zeros((nt + 1, 2, nx, nz), np.float32)
    C.check(L.fwi2d_propagate(kind, 0, C.ptr(mc), C.ptr(np.ascontiguousarray(g["src"])), C.ptr(rcv),
                              ctypes.byref(ji), ctypes.byref(jd), None, None, C.ptr(full), None, ctypes.byref(params),
                              1, nr, nx, nz, d, d))
    e_tr = K.rel_l2(rcv, g["rcv"])
    grad = np.zeros((3, nx, nz), np.float32)
    dummy = np.zeros((2, 1, nt), np.float32)
    C.check(L.fwi2d_propagate(kind, 1, C.ptr(mc), C.ptr(np.ascontiguousarray(g["adj"])), C.ptr(dummy),
                              ctypes.byref(jd), ctypes.byref(ji), None, None, C.ptr(full), C.ptr(grad),
                              ctypes.byref(params), 1, nr, nx, nz, d, d))
    e_g = K.rel_l2(grad, g["grad"])
    print("dipole receivers: traces rel-L2 %.3e (bitwise %.4f), gradient rel-L2 %.3e" % (
        e_tr, np.mean(rcv == g["rcv"]), e_g))
    assert e_tr <= 1e-6
    assert e_g <= 1e-5


def test_dipole_rejected_where_unsupported():
    g = dict(np.load(os.path.join(GOLD, "dipole_f32.npz")))
    nx, nz, d, nt = int(g["nx"]), int(g["nz"]), float(g["d"]), 20
    L = F.load()
    dip = dipole_tables(g["rx"], g["rz"], g["rdip"], float(g["gl"]), nx, nz, d, d)
    jd = C.Injector(C.INJ_DIPOLE, len(g["rx"]), C.ptr(dip[0]), C.ptr(dip[1]), C.ptr(dip[2]), C.ptr(dip[3]))
    m = np.ones((2, nx, nz), np.float32)
    params = F.make_params(**K.par_dict(nt=nt, dt=1e-3, sub=0))
    rcv = np.zeros((1, len(g["rx"]), nt), np.float32)
    src = np.zeros((1, 1, nt), np.float32)
    rc = L.fwi2d_propagate(F.ACOUSTIC, 0, C.ptr(m), C.ptr(src), C.ptr(rcv), ctypes.byref(jd), ctypes.byref(jd),
                           None, None, None, None, ctypes.byref(params), 1, len(g["rx"]), nx, nz, d, d)
    assert rc == -5 and b"dipole" in L.fwi2d_last_error()
