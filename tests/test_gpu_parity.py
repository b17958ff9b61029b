"""CUDA path vs the oracle on seeded small cases, through the C ABI.

The kernels restate the reference's single-precision operation order, so the
FP32 traces, snapshots and gradients are compared at a relative L2 tolerance
of 1e-6 (traces) / 1e-5 (gradients) -- tighter than the 1e-5 / 1e-4 parity
bar -- and the number of bitwise-equal samples is reported.
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from tests import cases as K

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-6
GRAD_TOL = 1e-5


def run_gpu(kind, mc, src, pd, nx, nz, d, src_locs, rcv_locs, adj_src=None, mt=0, shape=-1, prec=F.SNAP_FP32):
    P = F.Propagator(0)
    P.set_model(kind, mc, d, d)
    params = F.make_params(**pd, snapshot_precision=prec, tile_shape=shape)
    shot = F.ShotSpec(0, nx, pd["nt"], src_locs[0], src_locs[1], rcv_locs[0], rcv_locs[1], mt=bool(mt))
    P.set_shots(params, [shot])
    rcv = P.forward([src], store=True)[0]
    g = None
    if adj_src is not None:
        g = P.adjoint([adj_src])
    snaps = np.stack([P.snapshot(0, k) for k in range(0, pd["nt"], max(1, pd["nt"] // 5))])
    P.close()
    return rcv, g, snaps


@pytest.mark.parametrize("kind,mt,bc", [
    (O.KIND_ELASTIC, 0, (1, 2, 2, 2)),
    (O.KIND_ELASTIC, 0, (2, 2, 2, 2)),
    (O.KIND_ELASTIC, 0, (1, 1, 1, 1)),
    (O.KIND_ELASTIC, 1, (1, 2, 2, 2)),
    (O.KIND_VTI, 0, (1, 2, 2, 2)),
    (O.KIND_VTI, 0, (2, 2, 2, 2)),
])
@pytest.mark.parametrize("shape,grid", [(0, (72, 80)), (1, (72, 80)), (2, (72, 80)), (3, (72, 80)),
                                        (0, (120, 200)), (1, (120, 200)),
                                        (4, (72, 80)), (6, (120, 200)), (7, (120, 200)), (11, (120, 200)),
                                        (11, (60, 251)), (14, (72, 80)), (15, (72, 80)), (14, (120, 200)),
                                        (15, (60, 251)), (16, (120, 200)), (17, (120, 200)), (17, (60, 251))])
def test_forward_adjoint_vs_oracle(kind, mt, bc, shape, grid):
    """Shapes 0-3 run the tile kernel over the whole grid: small grids exercise
    the boundary path only; the 120 x 200 grid has interior tiles, which take
    the lean path of the 64-row tile shapes.  Shapes 4 and up run the
    marching kernel on the rows clear of the x boundary bands (one z window
    on 80 rows, two on 200; on 251 rows with 128-cell windows the last
    window is shifted up so that it owns the whole bottom band) and runs of
    64 or 32 rows.  Shapes 14 to 17 are framed plans: 32 x 8, 32 x 16, 64 x 8
    and 64 x 16 tiles on the tile kernel's interior paths (one cell, or a
    z-pair in packed FP32x2 arithmetic, per thread) over the cells clear of
    the bands (the last window of each axis flush with the band, owning part
    of its cells), the bands on the band kernels.  Tile shapes 0 and 1 on the
    200-row grid also run z-pair windows that own part of their cells."""
    nx, nz = grid
    d, nt = 0.01, 220 if nz < 100 else 160
    m = K.model_case(kind, nx, nz, d, seed=3)
    mc = K.converted(kind, m)
    sl, rl = K.geometry(nx, nz, d, nr=24)
    pd = K.par_dict(nt=nt, dt=1e-3, bc=bc, mt=mt)
    src = K.sources(3 if mt else 2, nt, 1e-3)
    port = O.Port(32)
    par = O.make_par(**pd, ns=1, nr=len(rl[0]))
    rcv_o, full_o = K.oracle_forward(port, kind, mc, src, par, nx, nz, d, sl, rl, mt=mt)
    adj = np.ascontiguousarray(rcv_o[:, :, ::-1])
    g_o = K.oracle_adjoint(port, kind, mc, adj, par, nx, nz, d, sl, rl, full_o, mt=mt)

    rcv_g, g_g, snaps = run_gpu(kind, mc, src, pd, nx, nz, d, sl, rl, adj_src=adj, mt=mt, shape=shape)
    e_tr = K.rel_l2(rcv_g, rcv_o)
    e_gr = K.rel_l2(g_g, g_o)
    idx = list(range(0, nt, max(1, nt // 5)))
    e_sn = K.rel_l2(snaps, full_o[idx])
    print("kind %d mt %d bc %s shape %d: traces %.3e (bitwise %.4f) snapshots %.3e gradient %.3e (bitwise %.4f)" % (
        kind, mt, bc, shape, e_tr, np.mean(rcv_g == rcv_o), e_sn, e_gr, np.mean(g_g == g_o)))
    assert e_tr <= TRACE_TOL
    assert e_sn <= TRACE_TOL
    for c in range(3):
        assert K.rel_l2(g_g[c], g_o[c]) <= GRAD_TOL, "gradient component %d" % c


@pytest.mark.parametrize("kind", [O.KIND_ELASTIC, O.KIND_VTI])
@pytest.mark.parametrize("shape", [0, 1, 3, 16, 17])
def test_deep_source_vs_oracle(kind, shape):
    """Source and receivers deep inside a 120 x 240 grid, so that the wave
    crosses the interior windows of every shape from the first steps: the
    z-pair windows of the 64-row shapes (packed FP32x2 arithmetic) and the
    framed plans' interior tiles, against the oracle over 200 steps."""
    nx, nz = 120, 240
    d, nt = 0.01, 200
    m = K.model_case(kind, nx, nz, d, seed=9)
    mc = K.converted(kind, m)
    sl, rl = K.geometry(nx, nz, d, nr=24, sz=(100 + 0.3) * d, rz=70 * d)
    pd = K.par_dict(nt=nt, dt=1e-3, bc=(1, 2, 2, 2))
    src = K.sources(2, nt, 1e-3)
    port = O.Port(32)
    par = O.make_par(**pd, ns=1, nr=len(rl[0]))
    rcv_o, full_o = K.oracle_forward(port, kind, mc, src, par, nx, nz, d, sl, rl)
    adj = np.ascontiguousarray(rcv_o[:, :, ::-1])
    g_o = K.oracle_adjoint(port, kind, mc, adj, par, nx, nz, d, sl, rl, full_o)
    rcv_g, g_g, snaps = run_gpu(kind, mc, src, pd, nx, nz, d, sl, rl, adj_src=adj, shape=shape)
    idx = list(range(0, nt, max(1, nt // 5)))
    e_tr, e_sn, e_gr = K.rel_l2(rcv_g, rcv_o), K.rel_l2(snaps, full_o[idx]), K.rel_l2(g_g, g_o)
    print("deep source kind %d shape %d: traces %.3e (bitwise %.4f) snapshots %.3e gradient %.3e (bitwise %.4f)" % (
        kind, shape, e_tr, np.mean(rcv_g == rcv_o), e_sn, e_gr, np.mean(g_g == g_o)))
    assert e_tr <= TRACE_TOL
    assert e_sn <= TRACE_TOL
    for c in range(3):
        assert K.rel_l2(g_g[c], g_o[c]) <= GRAD_TOL, "gradient component %d" % c


@pytest.mark.parametrize("bc", [(1, 2, 2, 2), (3, 3, 2, 2), (2, 2, 2, 2), (1, 1, 3, 3)])
@pytest.mark.parametrize("shape,grid", [(2, (72, 80)), (3, (72, 80)), (2, (120, 200)), (3, (60, 251))])
def test_acoustic_forward_adjoint_vs_oracle(bc, shape, grid):
    """Acoustic propagator (pressure, model (K, 1/rho)): pressure-release,
    absorbing and rigid sides; traces, snapshots and the (K, 1/rho) imaging
    condition against the oracle."""
    kind = O.KIND_ACOUSTIC
    nx, nz = grid
    d, nt = 0.01, 200
    mc = K.converted(kind, K.model_case(kind, nx, nz, d, seed=4))
    sl, rl = K.geometry(nx, nz, d, nr=20)
    pd = K.par_dict(nt=nt, dt=1e-3, bc=bc)
    src = K.sources(1, nt, 1e-3)
    port = O.Port(32)
    par = O.make_par(**pd, ns=1, nr=len(rl[0]))
    rcv_o, full_o = K.oracle_forward(port, kind, mc, src, par, nx, nz, d, sl, rl)
    adj = np.ascontiguousarray(rcv_o[:, :, ::-1])
    g_o = K.oracle_adjoint(port, kind, mc, adj, par, nx, nz, d, sl, rl, full_o)
    rcv_g, g_g, snaps = run_gpu(kind, mc, src, pd, nx, nz, d, sl, rl, adj_src=adj, shape=shape)
    e_tr = K.rel_l2(rcv_g, rcv_o)
    idx = list(range(0, nt, max(1, nt // 5)))
    e_sn = K.rel_l2(snaps, full_o[idx])
    print("acoustic bc %s shape %d: traces %.3e (bitwise %.4f) snapshots %.3e gradient %.3e / %.3e" % (
        bc, shape, e_tr, np.mean(rcv_g == rcv_o), e_sn, K.rel_l2(g_g[0], g_o[0]), K.rel_l2(g_g[1], g_o[1])))
    assert e_tr <= TRACE_TOL
    assert e_sn <= TRACE_TOL
    for c in range(2):
        assert K.rel_l2(g_g[c], g_o[c]) <= GRAD_TOL, "gradient component %d" % c


@pytest.mark.parametrize("kind", [O.KIND_ELASTIC, O.KIND_ACOUSTIC])
def test_dropin_propagate_matches_oracle(kind):
    """fwi2d_propagate: the propagate_gpu drop-in with the reference's buffers."""
    import ctypes
    nx, nz, d, nt = 64, 48, 0.01, 150
    nc = 1 if kind == O.KIND_ACOUSTIC else 2
    mc = K.converted(kind, K.model_case(kind, nx, nz, d, seed=5))
    sl, rl = K.geometry(nx, nz, d, nr=16)
    pd = K.par_dict(nt=nt, dt=1e-3)
    src = K.sources(nc, nt, 1e-3)
    port = O.Port(32)
    par = O.make_par(**pd, ns=1, nr=16)
    rcv_o, full_o = K.oracle_forward(port, kind, mc, src, par, nx, nz, d, sl, rl)
    adj = np.ascontiguousarray(rcv_o[:, :, ::-1])
    g_o = K.oracle_adjoint(port, kind, mc, adj, par, nx, nz, d, sl, rl, full_o)

    L = F.load()
    from fwi2d_b200 import _capi as C
    inj = F.injector_tables(0, sl[0], sl[1], nx, nz, d, d, 0, 0)
    ext = F.injector_tables(0, rl[0], rl[1], nx, nz, d, d, 0, 0)
    ji = C.Injector(0, 1, C.ptr(inj[0]), C.ptr(inj[1]), C.ptr(inj[2]), C.ptr(inj[3]))
    je = C.Injector(0, 16, C.ptr(ext[0]), C.ptr(ext[1]), C.ptr(ext[2]), C.ptr(ext[3]))
    params = F.make_params(**pd)
    rcv = np.zeros((nc, 16, nt), np.float32)
    full = np.zeros_like(full_o)
    C.check(L.fwi2d_propagate(kind, 0, C.ptr(mc), C.ptr(np.ascontiguousarray(src)), C.ptr(rcv), ctypes.byref(ji),
                              ctypes.byref(je), None, None, C.ptr(full), None, ctypes.byref(params), 1, 16, nx, nz, d, d))
    assert K.rel_l2(rcv, rcv_o) <= TRACE_TOL
    assert K.rel_l2(full, full_o) <= TRACE_TOL
    g = np.zeros((2 if kind == O.KIND_ACOUSTIC else 3, nx, nz), np.float32)
    dummy = np.zeros((nc, 1, nt), np.float32)
    C.check(L.fwi2d_propagate(kind, 1, C.ptr(mc), C.ptr(adj), C.ptr(dummy), ctypes.byref(je), ctypes.byref(ji),
                              None, None, C.ptr(full), C.ptr(g), ctypes.byref(params), 1, 16, nx, nz, d, d))
    assert K.rel_l2(g, g_o) <= GRAD_TOL
