"""The two forms of the boundary-band kernels of framed and marching plans.

A plan's frame (the 6-cell bands along every edge) runs on band kernels that
update a cell's two field components in one thread, or in two warps
(FWI2D_BAND_SPLIT=1, the default for plans with few band windows).  Both
forms follow the reference's operation order per component, so each is
compared with the oracle at the parity tolerances and with the other form
bitwise, on framed (14, 16) and marching (6) plans, every propagator that
has a frame, free-surface and absorbing tops, point and moment-tensor
sources.
"""
import numpy as np
import pytest

import oracle as O
from tests import cases as K
from tests.test_gpu_parity import GRAD_TOL, TRACE_TOL, run_gpu

pytestmark = pytest.mark.gpu


# source cell (x, z) in units of the cell size: in the left band, in the top
# band, or in the right band next to the bottom corner
LEFT, TOP, RIGHT_LOW = (2.3, 100.2), (60.1, 3.4), (116.2, 195.3)


@pytest.mark.parametrize("kind,mt,bc,at", [
    (O.KIND_ELASTIC, 0, (1, 2, 2, 2), LEFT),
    (O.KIND_ELASTIC, 0, (2, 2, 2, 2), TOP),
    (O.KIND_ELASTIC, 1, (1, 1, 1, 1), RIGHT_LOW),
    (O.KIND_VTI, 0, (1, 2, 2, 2), TOP),
    (O.KIND_VTI, 0, (2, 1, 1, 2), LEFT),
])
@pytest.mark.parametrize("shape", [14, 16, 6])
def test_band_forms_vs_oracle(monkeypatch, kind, mt, bc, at, shape):
    nx, nz = 120, 200
    d, nt = 0.01, 160
    m = K.model_case(kind, nx, nz, d, seed=5)
    mc = K.converted(kind, m)
    # a line of receivers across the grid, bands included, two cells above the source
    sl, rl = K.geometry(nx, nz, d, nr=24, sx=at[0] * d, sz=at[1] * d, rz=(at[1] - 2) * d)
    pd = K.par_dict(nt=nt, dt=1e-3, bc=bc, mt=mt)
    src = K.sources(3 if mt else 2, nt, 1e-3)
    port = O.Port(32)
    par = O.make_par(**pd, ns=1, nr=len(rl[0]))
    rcv_o, full_o = K.oracle_forward(port, kind, mc, src, par, nx, nz, d, sl, rl, mt=mt)
    adj = np.ascontiguousarray(rcv_o[:, :, ::-1])
    g_o = K.oracle_adjoint(port, kind, mc, adj, par, nx, nz, d, sl, rl, full_o, mt=mt)
    out = {}
    for split in ("0", "1"):
        monkeypatch.setenv("FWI2D_BAND_SPLIT", split)
        rcv_g, g_g, snaps = run_gpu(kind, mc, src, pd, nx, nz, d, sl, rl, adj_src=adj, mt=mt, shape=shape)
        e_tr, e_gr = K.rel_l2(rcv_g, rcv_o), K.rel_l2(g_g, g_o)
        print("split %s kind %d mt %d bc %s shape %d: traces %.3e (bitwise %.4f) gradient %.3e (bitwise %.4f)" % (
            split, kind, mt, bc, shape, e_tr, np.mean(rcv_g == rcv_o), e_gr, np.mean(g_g == g_o)))
        assert e_tr <= TRACE_TOL
        for c in range(3):
            assert K.rel_l2(g_g[c], g_o[c]) <= GRAD_TOL, "gradient component %d" % c
        out[split] = (rcv_g, g_g, snaps)
    for a, b in zip(out["0"], out["1"]):
        assert np.array_equal(a, b), "the two band forms differ"
