"""Reduced-precision snapshot storage against the FP64 oracle.

The forward snapshots the imaging condition reads can be kept in FP32, or in
BF16 / FP16 scaled per snapshot by a power of two chosen from the snapshot's
max |u|; the stencil arithmetic stays FP32.  Relative L2 errors of the traces
and of the (lambda, mu, rho) imaging condition against the oracle built in
FP64 (the reference's ENABLE_DOUBLE_PRECISION build, restated), for the tile
and the marching kernels.
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from tests import cases as K
from tests.test_gpu_parity import run_gpu

pytestmark = pytest.mark.gpu

# bar for each precision (the gradient; traces are FP32 in every case)
# FP32 storage: the single-precision arithmetic's own distance from FP64.
# FP16 (11-bit significand with the per-snapshot scale) keeps every component
# within 1e-3.  BF16 (8-bit significand) keeps mu and rho within 1e-3 but not
# lambda: its imaging term (div u)(div v) takes spatial differences of the
# stored field, which magnify the storage rounding (about 5e-3 here).
BARS = {F.SNAP_FP32: 1e-4, F.SNAP_BF16: 1e-2, F.SNAP_FP16: 1e-3}


@pytest.mark.parametrize("kind", [O.KIND_ELASTIC, O.KIND_VTI])
@pytest.mark.parametrize("shape", [3, 8])
def test_snapshot_precision_vs_fp64_oracle(kind, shape):
    nx, nz, d, nt = 120, 200, 0.01, 400
    m = K.model_case(kind, nx, nz, d, seed=9)
    mc64 = O.Port(64).convert_model(kind, m)
    mc32 = K.converted(kind, m)
    sl, rl = K.geometry(nx, nz, d, nr=24)
    pd = K.par_dict(nt=nt, dt=1e-3, bc=(1, 2, 2, 2))
    src = K.sources(2, nt, 1e-3)
    o64 = O.Port(64)
    par = O.make_par(**pd, ns=1, nr=len(rl[0]))
    rcv64, full64 = K.oracle_forward(o64, kind, mc64, src, par, nx, nz, d, sl, rl)
    adj = np.ascontiguousarray(rcv64[:, :, ::-1])
    g64 = K.oracle_adjoint(o64, kind, mc64, adj, par, nx, nz, d, sl, rl, full64)
    errs = {}
    for prec in (F.SNAP_FP32, F.SNAP_BF16, F.SNAP_FP16):
        rcv, g, _ = run_gpu(kind, mc32, src, pd, nx, nz, d, sl, rl, adj_src=adj.astype(np.float32), shape=shape,
                            prec=prec)
        e_tr = K.rel_l2(rcv, rcv64)
        e_g = [K.rel_l2(g[c], g64[c]) for c in range(3)]
        errs[prec] = (e_tr, max(e_g))
        print("kind %d shape %d snapshots %s: traces %.2e  gradient (lambda, mu, rho) %.2e %.2e %.2e" % (
            kind, shape, {0: "fp32", 1: "bf16", 2: "fp16"}[prec], e_tr, *e_g))
    for prec, (e_tr, e_g) in errs.items():
        assert e_tr <= 1e-4
        assert e_g <= BARS[prec]
