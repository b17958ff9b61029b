"""Batched shots with uneven apertures and record lengths in one plan.

Each shot runs on its own cropped subgrid of the model (columns [x0, x0+nx)),
with its own record length.  All shots share one CUDA graph per pass.  Every
shot is checked against the oracle run on the same cropped model with the
same nt:

* the shot's receivers to 1e-6 rel-L2;
* the model-grid gradient (the sum of the shots' imaging conditions scattered
  onto their columns) to 1e-5 rel-L2.

The tile kernel, the marching kernel and the framed tile plan (the last two
with their band kernels) are covered, for the elastic and VTI propagators.  The grid spacing is 2^-7 km and
every location sits on a binary fraction of a cell, so that the injector
weights computed from model coordinates (the batch) and from the cropped
grid's own coordinates (the oracle) are the same numbers.
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from tests import cases as K

pytestmark = pytest.mark.gpu

SHOTS = [  # x0, nx, nt, source x offset (cells), receivers
    (0, 72, 140, 30, 10),
    (20, 96, 121, 51, 14),
    (61, 80, 150, 20, 12),
    (100, 60, 97, 33, 8),
    (44, 116, 133, 70, 16),
]


@pytest.mark.parametrize("kind", [O.KIND_ELASTIC, O.KIND_VTI])
@pytest.mark.parametrize("shape", [3, 4, 14])
def test_uneven_batch_matches_per_shot_oracle(kind, shape):
    nxm, nz, d, dt = 160, 72, 2.0 ** -7, 1e-3
    raw = K.model_case(kind, nxm, nz, d, seed=21)
    mc = K.converted(kind, raw)
    nt_max = max(s[2] for s in SHOTS)
    pd = K.par_dict(nt=nt_max, dt=dt, bc=(1, 2, 2, 2), taper=(0, 8, 8, 8))
    specs, srcs, adjs, ref_rcv, ref_g = [], [], [], [], np.zeros((3, nxm, nz))
    port = O.Port(32)
    rng = np.random.default_rng(3)
    for x0, nx, nt, sxo, nr in SHOTS:
        sx = np.array([(x0 + sxo + 0.25) * d], np.float32)
        sz = np.array([2.5 * d], np.float32)
        step = (nx - 8) // nr
        rx = ((x0 + 3.25 + step * np.arange(nr)) * d).astype(np.float32)
        rz = np.full(nr, 2.25 * d, np.float32)
        specs.append(F.ShotSpec(x0, nx, nt, sx, sz, rx, rz))
        src = K.sources(2, nt, dt)
        srcs.append(src)
        # oracle on the cropped model, origin at the shot's first column
        par = O.make_par(**dict(pd, nt=nt), ns=1, nr=nr)
        mcs = np.ascontiguousarray(mc[:, x0:x0 + nx])
        sl = (sx - np.float32(x0 * d), sz)
        rl = (rx - np.float32(x0 * d), rz)
        rcv_o, full_o = K.oracle_forward(port, kind, mcs, src, par, nx, nz, d, sl, rl)
        adj = (rng.standard_normal(rcv_o.shape) * np.abs(rcv_o).max()).astype(np.float32)
        g_o = K.oracle_adjoint(port, kind, mcs, adj, par, nx, nz, d, sl, rl, full_o)
        ref_rcv.append(rcv_o)
        adjs.append(adj)
        ref_g[:, x0:x0 + nx] += g_o[:3]
    P = F.Propagator(0)
    P.set_model(kind, mc, d, d)
    P.set_shots(F.make_params(**pd, tile_shape=shape), specs)
    rcv = P.forward(srcs, store=True)
    g = P.adjoint(adjs)
    info = P.plan_info()
    P.close()
    errs = [K.rel_l2(a, b) for a, b in zip(rcv, ref_rcv)]
    e_g = K.rel_l2(g, ref_g)
    print("kind %d shape %d: receivers per shot %s, model-grid gradient %.2e (bitwise %.4f), launches %s" % (
        kind, shape, ["%.1e" % e for e in errs], e_g, np.mean(g == ref_g.astype(np.float32)), info))
    assert max(errs) <= 1e-6
    assert e_g <= 1e-5
