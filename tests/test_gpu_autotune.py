"""The tile-shape autotuner on a gradient plan large enough to be tuned
(>= 2e7 cell-steps): two shots of different record lengths, tile_shape = -1.

The tuner builds and times candidate plans (sampled forward windows, adjoint
steps, then whole forward + adjoint passes of the close candidates) before it
builds the plan it keeps.  FWI2D_TUNE_CLOSE = 100 sends every shape through
the whole-pass stage, so that stage runs here whatever the sampled scores.
The kept plan must behave exactly like a plan built directly with the chosen
shape: same gradient and misfit, bit for bit; and, since every shape restates
the same operation order, like a plan on another shape too.
"""
import numpy as np
import pytest

import fwi2d_b200 as F
from fwi2d_b200 import workloads as W
from tests import cases as K

pytestmark = pytest.mark.gpu


def _run(tile_shape):
    kind, nx, nz, d, dt = F.ELASTIC, 220, 130, 0.01, 1e-3
    nts = [460, 330]
    model = W.convert(kind, K.model_case(kind, nx, nz, d, seed=3))
    shots, srcs, obs = [], [], []
    rng = np.random.default_rng(4)
    for k, nt in enumerate(nts):
        sl, rl = K.geometry(nx, nz, d, nr=24, sx=(60 + 90 * k + 0.3) * d)
        shots.append(F.ShotSpec(0, nx, nt, sl[0], sl[1], rl[0], rl[1]))
        srcs.append(K.sources(2, nt, dt))
        obs.append((rng.standard_normal((2, 24, nt)) * 1e-3).astype(np.float32))
    assert sum(nx * nz * nt for nt in nts) >= 2e7   # large enough for the tuner
    P = F.Propagator(0)
    P.set_model(kind, model, d, d)
    P.set_shots(F.make_params(**K.par_dict(nt=max(nts), dt=dt, bc=(1, 2, 2, 2), taper=(0, 10, 10, 10)),
                              tile_shape=tile_shape), shots)
    shape = P.plan_info()["tile_shape"]
    g, f = P.fwi_gradient(model, srcs, obs)
    P.close()
    return shape, g, f


def test_autotuned_plan_equals_direct_plan(monkeypatch):
    monkeypatch.setenv("FWI2D_TUNE_CLOSE", "100")
    shape, g, f = _run(-1)
    assert shape >= 0
    shape2, g2, f2 = _run(shape)
    assert shape2 == shape
    assert np.array_equal(g, g2) and f == f2
    other = 3 if shape != 3 else 2
    _, g3, f3 = _run(other)
    err = K.rel_l2(g, g3)
    print("autotuned shape %d; vs shape %d: gradient rel-L2 %.3e, misfit %.9e vs %.9e" % (shape, other, err, f, f3))
    assert err <= 1e-6
    assert abs(f - f3) <= 1e-6 * abs(f3)
