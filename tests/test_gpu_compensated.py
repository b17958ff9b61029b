"""Compensated gradient accumulation (params.compensated = 1).

The imaging condition adds one term per time sample into every gradient
cell.  The reference sums them in single precision, one rounding per step
(we_op.cpp:505-562); the library does the same by default, bitwise.  With
`compensated` set, the step kernels sum the terms of 8 adjoint steps in
FP32 and each such partial sum joins a running (hi, lo) pair by Neumaier's
compensated summation.

The check isolates the summation: the oracle's test switch
(orc32_set_exact_gradient_sum) sums the same single-precision terms in
double and rounds once, the exact sum.  Against it, the compensated gradient
must be several times closer than the plain one (the floor is the final
rounding to FP32 that both share, about 6e-8 relative).  The checkpointed plan
(checkpoint-and-recompute) closes its windows after the same adjoint
launches, so it gives the same compensated gradient bitwise.  The error of
both against the FP64 oracle is reported.
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from tests import cases as K

pytestmark = pytest.mark.gpu


def _gpu_grad(kind, mc, src, adj, pd, nx, nz, d, sl, rl, **opts):
    P = F.Propagator(0)
    P.set_model(kind, mc, d, d)
    P.set_shots(F.make_params(**pd, **opts), [F.ShotSpec(0, nx, pd["nt"], sl[0], sl[1], rl[0], rl[1])])
    P.forward([src], store=True)
    g = P.adjoint([adj])
    P.close()
    return g


@pytest.mark.parametrize("kind", [O.KIND_ELASTIC, O.KIND_VTI])
def test_compensated_gradient_closer_to_exact_sum(kind):
    nx, nz, d, nt = 100, 80, 0.01, 3000
    raw = K.model_case(kind, nx, nz, d, seed=13)
    mc = K.converted(kind, raw)
    sl, rl = K.geometry(nx, nz, d, nr=20)
    pd = K.par_dict(nt=nt, dt=1e-3)
    src = K.sources(2, nt, 1e-3)
    port = O.Port(32)
    par = O.make_par(**pd, ns=1, nr=len(rl[0]))
    rcv_o, full_o = K.oracle_forward(port, kind, mc, src, par, nx, nz, d, sl, rl)
    rng = np.random.default_rng(4)
    adj = (rng.standard_normal(rcv_o.shape) * np.abs(rcv_o).max()).astype(np.float32)
    g_plain_o = K.oracle_adjoint(port, kind, mc, adj, par, nx, nz, d, sl, rl, full_o)
    port.lib.orc32_set_exact_gradient_sum(1)
    try:
        g_exact = K.oracle_adjoint(port, kind, mc, adj, par, nx, nz, d, sl, rl, full_o)
    finally:
        port.lib.orc32_set_exact_gradient_sum(0)
    del full_o
    p64 = O.Port(64)
    par64 = O.make_par(**pd, ns=1, nr=len(rl[0]))
    _, full64 = K.oracle_forward(p64, kind, mc, src, par64, nx, nz, d, sl, rl)
    g64 = K.oracle_adjoint(p64, kind, mc, adj, par64, nx, nz, d, sl, rl, full64)
    del full64

    g_plain = _gpu_grad(kind, mc, src, adj, pd, nx, nz, d, sl, rl, tile_shape=3)
    g_comp = _gpu_grad(kind, mc, src, adj, pd, nx, nz, d, sl, rl, tile_shape=3, compensated=1)
    g_comp_ck = _gpu_grad(kind, mc, src, adj, pd, nx, nz, d, sl, rl, tile_shape=3, compensated=1,
                          checkpoint_every=37)
    e_plain_bitwise = K.rel_l2(g_plain, g_plain_o)
    print("kind %d nt %d: plain vs oracle %.2e; vs exact sum: plain %s, compensated %s; vs FP64: plain %s, "
          "compensated %s" % (
              kind, nt, e_plain_bitwise,
              ["%.2e" % K.rel_l2(g_plain[c], g_exact[c]) for c in range(3)],
              ["%.2e" % K.rel_l2(g_comp[c], g_exact[c]) for c in range(3)],
              ["%.2e" % K.rel_l2(g_plain[c], g64[c]) for c in range(3)],
              ["%.2e" % K.rel_l2(g_comp[c], g64[c]) for c in range(3)]))
    assert e_plain_bitwise <= 1e-6
    assert np.array_equal(g_comp, g_comp_ck)
    for c in range(3):
        e_p, e_c = K.rel_l2(g_plain[c], g_exact[c]), K.rel_l2(g_comp[c], g_exact[c])
        assert e_p > 0, "component %d: the plain sum shows no rounding to measure" % c
        assert e_c <= 0.3 * e_p, "component %d: compensated %.3e vs plain %.3e" % (c, e_c, e_p)
        assert K.rel_l2(g_comp[c], g64[c]) <= 1.05 * K.rel_l2(g_plain[c], g64[c]) + 1e-9
