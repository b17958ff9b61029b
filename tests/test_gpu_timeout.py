"""Bounded device waits report their failure to the caller.

The marching kernel waits on an mbarrier for the bulk copies of each row.
Every such wait is bounded by a poll limit (FWI2D_SPIN_LIMIT, read when a plan
is built).  A wait that reaches it records the row in a device flag and keeps
waiting, again bounded, for the same copies, so that none is left in flight
in the CTA's shared memory (past that second bound the CTA leaves).  After
the pass the engine moves the flag into the plan's status word and the call
returns FWI2D_ERR_TIMEOUT instead of results nobody checked.

The test sets the limit to 0 polls, so every wait reaches it at once (the
second bound is the ordinary one, nothing is left spinning), checks the error
code and that the pass's snapshots are refused, and then shows that the
context still works: a plan built with the default limit on the same context
gives the oracle's traces.
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from fwi2d_b200 import _capi as C
from tests import cases as K

pytestmark = pytest.mark.gpu

MARCH_SHAPE = 11          # marching kernel, 128-cell z windows, runs of 32 rows


def _case():
    kind, nx, nz, d, nt = O.KIND_ELASTIC, 120, 200, 0.01, 120
    mc = K.converted(kind, K.model_case(kind, nx, nz, d, seed=11))
    sl, rl = K.geometry(nx, nz, d, nr=16)
    pd = K.par_dict(nt=nt, dt=1e-3)
    src = K.sources(2, nt, 1e-3)
    return kind, nx, nz, d, nt, mc, sl, rl, pd, src


def test_march_wait_limit_returns_timeout(monkeypatch):
    kind, nx, nz, d, nt, mc, sl, rl, pd, src = _case()
    P = F.Propagator(0)
    P.set_model(kind, mc, d, d)
    shot = F.ShotSpec(0, nx, nt, sl[0], sl[1], rl[0], rl[1])
    monkeypatch.setenv("FWI2D_SPIN_LIMIT", "0")
    P.set_shots(F.make_params(**pd, tile_shape=MARCH_SHAPE), [shot])
    with pytest.raises(C.Fwi2dError) as err:
        P.forward([src], store=True)
    assert err.value.code == C.ERR_TIMEOUT, str(err.value)
    assert "reached its limit" in str(err.value)
    # the adjoint refuses the snapshots of the failed pass
    with pytest.raises(C.Fwi2dError):
        P.adjoint([np.zeros((2, len(rl[0]), nt), np.float32)])

    # same context, default limit: a correct pass
    monkeypatch.delenv("FWI2D_SPIN_LIMIT")
    P.set_shots(F.make_params(**pd, tile_shape=MARCH_SHAPE), [shot])
    rcv = P.forward([src], store=False)[0]
    P.close()
    port = O.Port(32)
    par = O.make_par(**pd, ns=1, nr=len(rl[0]))
    rcv_o, _ = K.oracle_forward(port, kind, mc, src, par, nx, nz, d, sl, rl)
    assert K.rel_l2(rcv, rcv_o) <= 1e-6
