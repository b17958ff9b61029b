"""FWI gradients of batches whose snapshots do not fit the device at once.

When the snapshots of all shots of a plan exceed the device memory (less a
reserve), the plan splits its shots into waves: contiguous runs of shots
whose snapshots fit together.  Each wave has its own graphs over its shots'
work units; the waves share one snapshot store, and fwi2d_fwi_gradient runs
forward, residual and adjoint wave by wave, summing the gradient over all
shots.  FWI2D_SNAPSHOT_BUDGET replaces the budget so that a small batch
splits here.

Checks, for the elastic and VTI propagators on the tile and the marching
plans, and for the acoustic and acoustic-elastic propagators on their tile
plans: a batch of uneven shots (cropped grids, uneven record lengths) split
into three or more waves gives the same gradient and misfit as the same
batch in one wave, bitwise; its plan holds the snapshots of one wave only;
the forward without snapshots still runs every shot at once, while a forward
that stores snapshots of all shots is refused with FWI2D_ERR_UNSUPPORTED.
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from fwi2d_b200 import _capi as C
from tests import cases as K

pytestmark = pytest.mark.gpu

SHOTS = [  # x0, nx, nt, source x offset (cells), receivers
    (0, 72, 140, 30, 10),
    (20, 96, 121, 51, 14),
    (61, 80, 150, 20, 12),
    (100, 60, 97, 33, 8),
    (44, 116, 133, 70, 16),
    (10, 88, 111, 40, 12),
]


NZA = 14   # fluid rows of the acoustic-elastic batch


def _batch(kind):
    nxm, nz, d, dt = 160, 72, 2.0 ** -7, 1e-3
    ae = kind == O.KIND_AE
    mkind = O.KIND_ELASTIC if ae else kind
    raw = K.model_case(mkind, nxm, nz, d, seed=21)
    true = K.model_case(mkind, nxm, nz, d, seed=22)
    oz = (NZA - 1) * d
    specs, srcs = [], []
    for x0, nx, nt, sxo, nr in SHOTS:
        sx = np.array([(x0 + sxo + 0.25) * d], np.float32)
        sz = np.array([2.5 * d], np.float32)
        step = (nx - 8) // nr
        rx = ((x0 + 3.25 + step * np.arange(nr)) * d).astype(np.float32)
        rz = np.full(nr, 2.25 * d, np.float32)
        if ae:
            # source in the water; receivers below the seabed and in the water
            specs.append(F.ShotSpec(x0, nx, nt, [0.0], [oz], rx, rz + oz, water_src_x=sx, water_src_z=sz,
                                    water_rcv_x=rx, water_rcv_z=rz + d))
        else:
            specs.append(F.ShotSpec(x0, nx, nt, sx, sz, rx, rz))
        srcs.append(K.sources(1 if kind in (O.KIND_ACOUSTIC, O.KIND_AE) else 2, nt, dt))
    extra = dict(nza=NZA, acoustic_source=1) if ae else {}
    pd = K.par_dict(nt=max(s[2] for s in SHOTS), dt=dt, bc=(2, 2, 2, 2) if ae else (1, 2, 2, 2),
                    taper=(4, 8, 8, 8) if ae else (0, 8, 8, 8), **extra)
    return raw, true, specs, srcs, pd, d


def _gradient(kind, raw, true, specs, srcs, pd, d, shape):
    P = F.Propagator(0)
    mkind = O.KIND_ELASTIC if kind == O.KIND_AE else kind
    oz = (NZA - 1) * d if kind == O.KIND_AE else 0.0
    P.set_model(kind, K.converted(mkind, true), d, d, 0.0, oz)
    P.set_shots(F.make_params(**pd, tile_shape=shape), specs)
    obs = P.forward(srcs, store=False)
    mc = K.converted(mkind, raw)
    g, phi = P.fwi_gradient(mc, srcs, obs)
    info = P.plan_info()
    return P, g, phi, info


@pytest.mark.parametrize("kind,shape", [(O.KIND_ELASTIC, 3), (O.KIND_ELASTIC, 8), (O.KIND_VTI, 3), (O.KIND_VTI, 8),
                                        (O.KIND_ACOUSTIC, 3), (O.KIND_AE, 3)])
def test_waves_match_one_wave(kind, shape, monkeypatch):
    raw, true, specs, srcs, pd, d = _batch(kind)
    P1, g1, phi1, info1 = _gradient(kind, raw, true, specs, srcs, pd, d, shape)
    P1.close()
    # about two shots' snapshots per wave
    monkeypatch.setenv("FWI2D_SNAPSHOT_BUDGET", str(info1["snapshot_bytes"] // 3))
    Pw, gw, phiw, infow = _gradient(kind, raw, true, specs, srcs, pd, d, shape)
    print("kind %d shape %d: one wave %s, waves %s, gradient bitwise %s, misfit %.9e / %.9e" % (
        kind, shape, info1, infow, np.array_equal(g1, gw), phi1, phiw))
    assert infow["snapshot_bytes"] <= info1["snapshot_bytes"] // 2
    assert np.array_equal(g1, gw)
    assert phi1 == phiw
    # a forward that keeps the snapshots of every shot is refused; without them it runs
    with pytest.raises(C.Fwi2dError) as err:
        Pw.forward(srcs, store=True)
    assert err.value.code == C.ERR_UNSUPPORTED
    assert "waves" in str(err.value)
    Pw.forward(srcs, store=False)
    Pw.close()
