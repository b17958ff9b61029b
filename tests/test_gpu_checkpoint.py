"""Checkpoint-and-recompute (params.checkpoint_every = K > 0).

The forward keeps checkpoints of the two field buffers every K steps and no
snapshots.  The adjoint replays each segment from its checkpoint, storing that
segment's snapshots in a window of K + 2 slots, and then runs the segment's
adjoint steps.  The replay repeats the forward launches exactly, so:

* receivers equal the stored-snapshot run's, bitwise;
* the imaging condition also equals it bitwise, for every K (K = 1, uneven last
  segments, K >= nt), every propagator, tile and marching kernels, and FP32 and
  16-bit snapshot storage.
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from fwi2d_b200 import _capi as C
from tests import cases as K

pytestmark = pytest.mark.gpu


def _run(kind, shape, prec, ckpt, nx, nz, nt, nshots=2, seed=0):
    d = 0.01
    m = K.converted(kind, K.model_case(kind, nx, nz, d, seed))
    P = F.Propagator(0)
    P.set_model(kind, m, d, d)
    pd = K.par_dict(nt=nt, dt=1e-3)
    params = F.make_params(**pd, snapshot_precision=prec, tile_shape=shape, checkpoint_every=ckpt)
    shots = []
    for s in range(nshots):
        (sx, sz), (rx, rz) = K.geometry(nx, nz, d, sx=(0.3 + 0.4 * s) * (nx - 1) * d + 0.3 * d)
        shots.append(F.ShotSpec(0, nx, nt, sx, sz, rx, rz))
    P.set_shots(params, shots)
    nc = P.ncomp()
    src = K.ricker(nt, 1e-3, 15.0, 0.05)
    srcs = [np.stack([src, src])[:nc].reshape(nc, 1, nt)] * nshots
    rcv = P.forward(srcs, store=True)
    rng = np.random.default_rng(seed + 7)
    adj = [rng.standard_normal(r.shape).astype(np.float32) for r in rcv]
    g = P.adjoint(adj)
    info = P.plan_info()
    P.close()
    return rcv, g, info


CASES = [
    (O.KIND_ELASTIC, 3, F.SNAP_FP32, (72, 80)),
    (O.KIND_ELASTIC, 3, F.SNAP_FP16, (72, 80)),
    (O.KIND_ELASTIC, 4, F.SNAP_FP32, (72, 80)),      # marching kernel + boundary bands
    (O.KIND_ELASTIC, 4, F.SNAP_BF16, (72, 80)),
    (O.KIND_VTI, 0, F.SNAP_FP32, (72, 80)),
    (O.KIND_VTI, 4, F.SNAP_FP16, (72, 80)),
    (O.KIND_ACOUSTIC, 2, F.SNAP_FP32, (72, 80)),
    (O.KIND_ACOUSTIC, 3, F.SNAP_FP16, (72, 80)),
    (O.KIND_ELASTIC, 14, F.SNAP_FP16, (72, 80)),     # framed plans: interior windows + frame kernels
    (O.KIND_VTI, 14, F.SNAP_FP32, (72, 80)),
    (O.KIND_ELASTIC, 16, F.SNAP_FP32, (72, 100)),
]


@pytest.mark.parametrize("kind,shape,prec,grid", CASES)
@pytest.mark.parametrize("every", [1, 7, 16, 200])
def test_checkpointed_gradient_equals_stored(kind, shape, prec, grid, every):
    nx, nz = grid
    nt = 61
    r0, g0, i0 = _run(kind, shape, prec, 0, nx, nz, nt)
    r1, g1, i1 = _run(kind, shape, prec, every, nx, nz, nt)
    for a, b in zip(r0, r1):
        assert np.array_equal(a, b)
    assert np.isfinite(g0).all() and np.abs(g0).max() > 0
    mism = np.mean(g0 != g1)
    print("kind %d shape %d prec %d every %d: %.4f of gradient samples differ; snapshot bytes %d -> %d" % (
        kind, shape, prec, every, mism, i0["snapshot_bytes"], i1["snapshot_bytes"]))
    assert np.array_equal(g0, g1)


def test_checkpointed_fwi_gradient_equals_stored():
    from fwi2d_b200 import workloads as W
    out = []
    for every in (0, 25):
        wl = W.elastic_single(nt=301)
        kind = wl["kind"]
        P = F.Propagator(0)
        P.set_model(kind, W.convert(kind, wl["start"]), wl["d"], wl["d"])
        s = wl["shots"][0]
        P.set_shots(F.make_params(**dict(wl["params"], checkpoint_every=every, snapshot_precision=F.SNAP_FP16)),
                    [F.ShotSpec(s["x0"], s["nx"], s["nt"], s["sx"], s["sz"], s["rx"], s["rz"])])
        src = [np.ascontiguousarray(wl["src"][:, :, :s["nt"]])]
        P.update_model(W.convert(kind, wl["true"]))
        obs = [P.forward(src, store=False)[0] * np.float32(0.9)]
        P.update_model(W.convert(kind, wl["start"]))
        g, phi = P.fwi_gradient(None, src, obs, seismotype=0)
        out.append((g, phi, P.plan_info()["snapshot_bytes"]))
        P.close()
    (g0, f0, b0), (g1, f1, b1) = out
    print("misfit %.9e / %.9e, device bytes %d -> %d" % (f0, f1, b0, b1))
    assert f0 == f1
    assert np.array_equal(g0, g1)
    assert b1 < b0


def test_checkpointing_needs_equal_record_lengths():
    kind = O.KIND_ELASTIC
    nx, nz, d = 72, 80, 0.01
    P = F.Propagator(0)
    P.set_model(kind, K.converted(kind, K.model_case(kind, nx, nz, d)), d, d)
    (sx, sz), (rx, rz) = K.geometry(nx, nz, d)
    shots = [F.ShotSpec(0, nx, 61, sx, sz, rx, rz), F.ShotSpec(0, nx, 50, sx, sz, rx, rz)]
    with pytest.raises(C.Fwi2dError) as e:
        P.set_shots(F.make_params(**K.par_dict(nt=61, dt=1e-3), checkpoint_every=10), shots)
    assert e.value.code == -5
    with pytest.raises(C.Fwi2dError) as e:
        P.set_shots(F.make_params(**K.par_dict(nt=61, dt=1e-3, sub=2), checkpoint_every=10), shots[:1])
    assert e.value.code == -1
    P.close()
