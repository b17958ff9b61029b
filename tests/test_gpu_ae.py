"""Acoustic-elastic propagator (nl_we_op_ae, src/cpp/we_op.cpp:2137-2577) on the GPU.

A homogeneous fluid layer of nza rows, with depths 0 .. oz, sits on the
elastic grid whose first row is at depth oz.  Each step on the GPU runs:

* the fluid layer (acoustic kernel: the reference's top, left and right
  conditions, a Neumann interface applied last);
* the elastic grid (tile kernel: version-1 lambda split, traction-free
  interface SAT applied last);
* the implicit coupling of the potential and uz at the interface, then that
  row's taper.

Checks against the reference's own outputs (tests/golden/acoustic_elastic_f32.npz)
and against the oracle on further cases, through the C ABI:

* traces ([fluid, x, z] blocks) and snapshots within 1e-6 rel-L2;
* the imaging condition within 1e-5;
* the number of bitwise-equal samples is printed.
"""
import os

import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from tests import cases as K

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _run(mc, src, pd, nx, nz, d, oz, sl, rx, rz_e, rz_w, wsrc, adj_src=None, shape=-1, prec=F.SNAP_FP32,
         snap_idx=()):
    P = F.Propagator(0)
    P.set_model(O.KIND_AE, mc, d, d, 0.0, oz)
    P.set_shots(F.make_params(**pd, tile_shape=shape, snapshot_precision=prec),
                [F.ShotSpec(0, nx, pd["nt"], sl[0], sl[1], rx, rz_e, water_src_x=wsrc[0], water_src_z=wsrc[1],
                            water_rcv_x=rx, water_rcv_z=rz_w)])
    rcv = P.forward([src], store=True)[0]
    g = P.adjoint([adj_src]) if adj_src is not None else None
    snaps = np.stack([P.snapshot(0, int(k)) for k in snap_idx]) if len(snap_idx) else None
    P.close()
    return rcv, g, snaps


def _oracle(prec, mc, src, pd, nx, nz, d, oz, sl, rx, rz_e, rz_w, wsrc, acoustic_source):
    o = O.Port(prec)
    nt = pd["nt"]
    par = O.make_par(**pd, ns=1, nr=len(rx))
    rcv = np.zeros((3, len(rx), nt), o.dtype)
    full = np.zeros((nt + 1, 2, nx, nz), o.dtype)
    o.propagate(O.KIND_AE, 0, o.arr(mc), o.arr(src), rcv, par, nx, nz, d, d, 0.0, oz,
                None if acoustic_source else sl, (rx, rz_e), full=full, water_inj_locs=wsrc,
                water_ext_locs=(rx, rz_w))
    adj = np.ascontiguousarray(rcv[:, :, ::-1])
    g = np.zeros((3, nx, nz), o.dtype)
    srcb = np.zeros((src.shape[0], 1, nt), o.dtype)
    o.propagate(O.KIND_AE, 1, o.arr(mc), adj, srcb, par, nx, nz, d, d, 0.0, oz, (rx, rz_e),
                None if acoustic_source else sl, full=full, grad=g, water_inj_locs=wsrc, water_ext_locs=(rx, rz_w))
    return rcv, g, full, adj


@pytest.mark.parametrize("shape", [2, 3])
def test_ae_matches_reference_golden(shape):
    g = dict(np.load(os.path.join(GOLD, "acoustic_elastic_f32.npz")))
    nx, nz, nt, d, oz, nza = int(g["nx"]), int(g["nz"]), int(g["nt"]), float(g["d"]), float(g["oz"]), int(g["nza"])
    pd = K.par_dict(nt=nt, dt=1e-3, bc=(1, 2, 2, 2), taper=(0, 6, 6, 6), nza=nza, acoustic_source=1)
    wsrc = (g["wsrc_x"], g["wsrc_z"])
    sl = (np.array([0.0], np.float32), np.array([oz], np.float32))
    adj = np.ascontiguousarray(g["rcv"][:, :, ::-1])
    rcv, grad, snaps = _run(g["model"], g["src"], pd, nx, nz, d, oz, sl, g["rcv_x"], g["rcv_ze"], g["rcv_zw"], wsrc,
                            adj_src=adj, shape=shape, snap_idx=g["snap_idx"])
    e_tr, e_sn, e_g = K.rel_l2(rcv, g["rcv"]), K.rel_l2(snaps, g["snaps"]), K.rel_l2(grad, g["grad"])
    print("AE shape %d vs reference: traces %.2e (bitwise %.4f)  snapshots %.2e  gradient %.2e (bitwise %.4f)" % (
        shape, e_tr, np.mean(rcv == g["rcv"]), e_sn, e_g, np.mean(grad == g["grad"])))
    assert e_tr <= 1e-6 and e_sn <= 1e-6
    assert e_g <= 1e-5


@pytest.mark.parametrize("bc,acoustic_source,grid", [
    ((1, 2, 2, 2), 1, (72, 80, 20)),
    ((2, 2, 2, 2), 1, (72, 80, 20)),
    ((3, 1, 1, 1), 1, (60, 44, 14)),
    ((1, 2, 2, 2), 0, (72, 80, 20)),
    ((2, 1, 2, 1), 0, (90, 72, 41)),
])
def test_ae_vs_oracle(bc, acoustic_source, grid):
    nx, nz, nza = grid
    d, nt = 0.01, 150
    oz = (nza - 1) * d
    raw = K.model_case(O.KIND_ELASTIC, nx, nz, d, seed=5)
    raw[0] += 0.5
    raw[1] = raw[0] / 1.8
    mc = K.converted(O.KIND_ELASTIC, raw)
    pd = K.par_dict(nt=nt, dt=1e-3, bc=bc, taper=(4, 8, 8, 8), nza=nza, acoustic_source=acoustic_source)
    rx = np.linspace(0.05, (nx - 5) * d, 16).astype(np.float32)
    rz_w = np.full(16, 0.03, np.float32)
    rz_e = np.full(16, oz + 0.02, np.float32)
    wsrc = (np.array([0.43 * nx * d], np.float32), np.array([0.052], np.float32))
    sl = (np.array([0.57 * nx * d], np.float32), np.array([oz + 0.061], np.float32))
    ncs = 1 if acoustic_source else 2
    src = K.sources(ncs, nt, 1e-3, f0=20.0, t0=0.05).astype(np.float32).reshape(ncs, 1, nt)
    r64, g64, _, _ = _oracle(64, mc.astype(np.float64), src.astype(np.float64), pd, nx, nz, d, oz, sl, rx, rz_e, rz_w,
                             wsrc, acoustic_source)
    r32, g32, full32, adj32 = _oracle(32, mc, src, pd, nx, nz, d, oz, sl, rx, rz_e, rz_w, wsrc, acoustic_source)
    rcv, grad, snaps = _run(mc, src, pd, nx, nz, d, oz, sl, rx, rz_e, rz_w, wsrc, adj_src=adj32,
                            snap_idx=[0, nt // 2, nt - 1])
    e_tr, e_g = K.rel_l2(rcv, r32), K.rel_l2(grad, g32)
    e_sn = K.rel_l2(snaps, full32[[0, nt // 2, nt - 1]])
    print("AE bc %s fluid source %d grid %s: traces %.2e (bitwise %.4f)  snapshots %.2e  gradient %.2e (bitwise %.4f)"
          "  [FP32 oracle vs FP64: traces %.2e]" % (bc, acoustic_source, grid, e_tr, np.mean(rcv == r32), e_sn, e_g,
                                                    np.mean(grad == g32), K.rel_l2(r32, r64)))
    assert np.abs(rcv).max() > 0 and np.abs(grad).max() > 0
    assert e_tr <= 1e-6 and e_sn <= 1e-6
    assert e_g <= 1e-5


def test_ae_dropin_propagate_matches_reference_golden():
    """fwi2d_propagate with the acoustic-elastic kind: the reference's
    per-shot buffers ([fluid, x, z] traces, [nt+1][2][nx][nz] snapshots) and
    the fluid injectors as inja / exta."""
    import ctypes
    from fwi2d_b200 import _capi as C
    g = dict(np.load(os.path.join(GOLD, "acoustic_elastic_f32.npz")))
    nx, nz, nt, d, oz, nza = int(g["nx"]), int(g["nz"]), int(g["nt"]), float(g["d"]), float(g["oz"]), int(g["nza"])
    pd = K.par_dict(nt=nt, dt=1e-3, bc=(1, 2, 2, 2), taper=(0, 6, 6, 6), nza=nza, acoustic_source=1)
    nr = len(g["rcv_x"])
    erc = F.injector_tables(0, g["rcv_x"], g["rcv_ze"], nx, nz, d, d, 0.0, oz)
    wrc = F.injector_tables(0, g["rcv_x"], g["rcv_zw"], nx, nza, d, d, 0.0, 0.0)
    wsr = F.injector_tables(0, g["wsrc_x"], g["wsrc_z"], nx, nza, d, d, 0.0, 0.0)

    def inj(t):
        return C.Injector(0, len(t[0]), C.ptr(t[0]), C.ptr(t[1]), C.ptr(t[2]), C.ptr(t[3]))
    je, jw, js = inj(erc), inj(wrc), inj(wsr)
    L = F.load()
    params = F.make_params(**pd)
    rcv = np.zeros((3, nr, nt), np.float32)
    full = np.zeros((nt + 1, 2, nx, nz), np.float32)
    C.check(L.fwi2d_propagate(O.KIND_AE, 0, C.ptr(g["model"]), C.ptr(np.ascontiguousarray(g["src"])), C.ptr(rcv),
                              None, ctypes.byref(je), ctypes.byref(js), ctypes.byref(jw), C.ptr(full), None,
                              ctypes.byref(params), 1, nr, nx, nz, d, d))
    assert np.array_equal(rcv, g["rcv"])
    assert np.array_equal(full[g["snap_idx"]], g["snaps"])
    adj = np.ascontiguousarray(g["rcv"][:, :, ::-1])
    grad = np.zeros((3, nx, nz), np.float32)
    dummy = np.zeros((1, 1, nt), np.float32)
    C.check(L.fwi2d_propagate(O.KIND_AE, 1, C.ptr(g["model"]), C.ptr(adj), C.ptr(dummy), ctypes.byref(je), None,
                              ctypes.byref(jw), ctypes.byref(js), C.ptr(full), C.ptr(grad), ctypes.byref(params), 1, nr,
                              nx, nz, d, d))
    print("AE drop-in gradient: bitwise %.4f, rel-L2 %.2e" % (np.mean(grad == g["grad"]), K.rel_l2(grad, g["grad"])))
    assert K.rel_l2(grad, g["grad"]) <= 1e-5


def test_ae_fwi_gradient_matches_reference_solver():
    """fwi2d_fwi_gradient on the acoustic-elastic propagator against the
    reference solver's gradient (nl_we_op_ae through nl_we_op_e's
    apply_forward / apply_jacobianT, fluid traces -Dt of the potential),
    tests/golden/fwi_gradient_ae_f32.npz."""
    from fwi2d_b200 import workloads as W
    g = dict(np.load(os.path.join(GOLD, "fwi_gradient_ae_f32.npz")))
    nx, nz, d, nt, dt, nza, oz = (int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nt"]), float(g["dt"]),
                                  int(g["nza"]), float(g["oz"]))
    P = F.Propagator(0)
    P.set_model(O.KIND_AE, W.convert(O.KIND_ELASTIC, g["start"]), d, d, 0.0, oz)
    pd = K.par_dict(nt=nt, dt=dt, bc=(2, 2, 2, 2), taper=(4, 10, 10, 10), nza=nza, acoustic_source=1)
    P.set_shots(F.make_params(**pd, tile_shape=3),
                [F.ShotSpec(0, nx, nt, [0.0], [oz], g["rx"], g["rz"], water_src_x=[float(g["sx"])],
                            water_src_z=[float(g["sz"])], water_rcv_x=g["rx"], water_rcv_z=g["rzw"])])
    grad, phi = P.fwi_gradient(W.convert(O.KIND_ELASTIC, g["start"]), [g["src"]], [g["obs"]], seismotype=1)
    P.close()
    err = K.rel_l2(grad, g["grad"])
    print("AE FWI gradient vs reference solver: rel-L2 %.3e (bitwise %.4f), misfit %.9e vs %.9e" % (
        err, np.mean(grad == g["grad"]), phi, float(g["misfit"])))
    assert err <= 1e-4
    assert abs(phi - float(g["misfit"])) <= 1e-5 * float(g["misfit"])


def test_ae_fwi_gradient_resampled_matches_reference_solver():
    """As above with the source and the data sampled at 2.5 ms and the
    propagation at 1 ms (sinc resampler, fwi2d_set_data_axis): the fluid
    traces' sign and the rate ratio on the data axis,
    tests/golden/fwi_gradient_ae_resampled_f32.npz."""
    from fwi2d_b200 import workloads as W
    g = dict(np.load(os.path.join(GOLD, "fwi_gradient_ae_resampled_f32.npz")))
    nx, nz, d, nt, dt, nza, oz = (int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nt"]), float(g["dt"]),
                                  int(g["nza"]), float(g["oz"]))
    nd, dd = int(g["nd"]), float(g["dd"])
    assert F.prop_nt(nd, dd, dt) == nt
    P = F.Propagator(0)
    P.set_model(O.KIND_AE, W.convert(O.KIND_ELASTIC, g["start"]), d, d, 0.0, oz)
    pd = K.par_dict(nt=nt, dt=dt, bc=(2, 2, 2, 2), taper=(4, 10, 10, 10), nza=nza, acoustic_source=1)
    P.set_shots(F.make_params(**pd, tile_shape=3),
                [F.ShotSpec(0, nx, nt, [0.0], [oz], g["rx"], g["rz"], water_src_x=[float(g["sx"])],
                            water_src_z=[float(g["sz"])], water_rcv_x=g["rx"], water_rcv_z=g["rzw"])])
    P.set_data_axis(dd, [nd], resampling="sinc")
    grad, phi = P.fwi_gradient(W.convert(O.KIND_ELASTIC, g["start"]), [g["src"]], [g["obs_sinc"]], seismotype=1)
    P.close()
    err = K.rel_l2(grad, g["grad_sinc"])
    mis = float(g["misfit_sinc"])
    print("AE FWI gradient, resampled data: rel-L2 %.3e (bitwise %.4f), misfit %.9e vs %.9e" % (
        err, np.mean(grad == g["grad_sinc"]), phi, mis))
    assert err <= 1e-4
    assert abs(phi - mis) <= 1e-5 * mis
