"""Host-API behaviour on the GPU: a model update keeps the plan valid.

``fwi2d_update_model`` re-uploads the model and recomputes the absorbing
boundary divisors and initial-injection scales of an existing plan.  Its
forward and adjoint must equal those of a fresh plan built on the new model,
bitwise, for every propagator.
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from tests import cases as K

pytestmark = pytest.mark.gpu


def _plan(kind, mc, nx, nz, d, nt, pd, shot, oz=0.0):
    P = F.Propagator(0)
    P.set_model(kind, mc, d, d, 0.0, oz)
    P.set_shots(F.make_params(**pd, tile_shape=3), [shot])
    return P


@pytest.mark.parametrize("kind", [O.KIND_ELASTIC, O.KIND_VTI, O.KIND_ACOUSTIC, O.KIND_AE])
def test_update_model_equals_fresh_plan(kind):
    nx, nz, d, nt = 64, 48, 0.01, 120
    ae = kind == O.KIND_AE
    base = O.KIND_ELASTIC if ae else kind
    ma = K.converted(base, K.model_case(base, nx, nz, d, seed=1))
    mb = K.converted(base, K.model_case(base, nx, nz, d, seed=2))
    (sx, sz), (rx, rz) = K.geometry(nx, nz, d, nr=10)
    pd = K.par_dict(nt=nt, dt=1e-3, bc=(2, 2, 2, 2))
    oz = 0.0
    shot = F.ShotSpec(0, nx, nt, sx, sz, rx, rz)
    if ae:
        nza = 14
        oz = (nza - 1) * d
        pd.update(nza=nza, acoustic_source=1)
        shot = F.ShotSpec(0, nx, nt, sx, sz + oz, rx, rz + oz, water_src_x=[0.31], water_src_z=[0.05],
                          water_rcv_x=rx, water_rcv_z=np.full(len(rx), 0.03, np.float32))
    ns = 1 if kind == O.KIND_ACOUSTIC or ae else 2
    src = K.sources(ns, nt, 1e-3).reshape(ns, 1, nt)
    P1 = _plan(kind, ma, nx, nz, d, nt, pd, shot, oz)
    P1.update_model(mb)
    r1 = P1.forward([src], store=True)[0]
    adj = np.ascontiguousarray(r1[:, :, ::-1])
    g1 = P1.adjoint([adj])
    P1.close()
    P2 = _plan(kind, mb, nx, nz, d, nt, pd, shot, oz)
    r2 = P2.forward([src], store=True)[0]
    g2 = P2.adjoint([adj])
    P2.close()
    assert np.abs(r2).max() > 0
    assert np.array_equal(r1, r2)
    assert np.array_equal(g1, g2)
