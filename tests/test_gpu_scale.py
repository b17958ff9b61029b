"""Parity at the benchmark configurations' own geometry, against the
reference's CPU build (oracle/_ref, the reference's sources compiled by
oracle/build_ref.sh and run with OpenMP on the host cores).

* single-shot elastic geometry (401 x 801 at 5 m, 400 two-component
  receivers every 10 m at 10 m depth, free surface on top, 60-cell tapers and
  absorbing sides, Ricker 10 Hz, dt = 0.4 ms), shortened to nt = 1000, on the
  plan the autotuner picks: forward traces, the last snapshot and the adjoint
  imaging condition (the reversed traces as adjoint sources).  The relative L2
  at the last time sample is reported too, since rounding drift grows with nt;
* the whole FWI gradient (fwi2d_fwi_gradient: forward, residual, adjoint
  sources, adjoint, quadrature, chain rule) against the reference solver's
  (nl_we_op_e::apply_forward + apply_jacobianT on the applyHt-weighted
  residual, optimization.hpp:760-890) on the same geometry at nt = 600, true
  model vs the smoothed starting model;
* four shots of the batch geometry (60 m spacing, 1.0-3.5 km apertures on
  cropped grids, uneven record lengths, shortened 8x) in one plan on the
  marching kernel's 224 x 32 units, against per-shot reference runs on the
  same cropped models;
* a checkpointed gradient (checkpoint-and-recompute every 200 steps) on a
  crop of the large-grid configuration (301 x 1001 at 2.5 m, Ricker 15 Hz,
  dt = 0.2 ms, nt = 2001) against the reference build.

Bars: the north-star parity bar, traces to 1e-5 and gradients to 1e-4
relative L2 (the kernels restate the reference's operation order, so the
measured errors are at or near 0).
"""
import numpy as np
import pytest

import oracle as O
import fwi2d_b200 as F
from fwi2d_b200 import workloads as W
from tests import cases as K

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.have_reference(32), reason="reference build (oracle/_ref) not present")]

TRACE_TOL = 1e-5
GRAD_TOL = 1e-4


def _par(params, nr):
    keys = ("nt", "sub", "dt", "bc_top", "bc_bottom", "bc_left", "bc_right", "taper_top", "taper_bottom",
            "taper_left", "taper_right", "taper_strength")
    return O.make_par(**{k: params[k] for k in keys}, ns=1, nr=nr)


def _ref_forward_adjoint(lib, kind, mc, src, adj_fn, par, nx, nz, d, sl, rl):
    rcv, full = K.oracle_forward(lib, kind, mc, src, par, nx, nz, d, sl, rl)
    adj = adj_fn(rcv)
    g = K.oracle_adjoint(lib, kind, mc, adj, par, nx, nz, d, sl, rl, full)
    return rcv, full[par.nt - 1].copy(), adj, g


def _vertical_force(nt, dt, f0=10.0):
    w = W.ricker(nt, dt, f0, 0.1)
    ang = np.float32(1.5708)
    return np.ascontiguousarray(np.stack([w * np.float32(np.cos(ang)), w * np.float32(np.sin(ang))])[:, None, :],
                                np.float32)


def test_single_shot_geometry_vs_reference_build():
    nt = 1000
    wl = W.elastic_single(nt=nt)
    kind, nx, nz, d = wl["kind"], wl["nx"], wl["nz"], wl["d"]
    mc = W.convert(kind, wl["start"])
    sh = wl["shots"][0]
    sl = (np.array(sh["sx"], np.float32), np.array(sh["sz"], np.float32))
    rl = (sh["rx"], sh["rz"])
    src = wl["src"]
    ref = O.Reference(32)
    par = _par(wl["params"], len(sh["rx"]))
    rcv_r, last_r, adj, g_r = _ref_forward_adjoint(
        ref, kind, mc, src, lambda r: np.ascontiguousarray(r[:, :, ::-1] * np.float32(1e3)), par, nx, nz, d, sl, rl)

    P = F.Propagator(0)
    P.set_model(kind, mc, d, d)
    P.set_shots(F.make_params(**wl["params"], tile_shape=-1),
                [F.ShotSpec(0, nx, nt, sh["sx"], sh["sz"], sh["rx"], sh["rz"])])
    rcv = P.forward([src], store=True)[0]
    last = P.snapshot(0, nt - 1)
    g = P.adjoint([adj])
    info = P.plan_info()
    P.close()
    e_tr, e_last = K.rel_l2(rcv, rcv_r), K.rel_l2(rcv[..., -1], rcv_r[..., -1])
    e_sn, e_g = K.rel_l2(last, last_r), K.rel_l2(g, g_r)
    print("401x801 nt=%d shape %s: traces %.2e (last sample %.2e, bitwise %.4f), last snapshot %.2e, "
          "gradient %.2e (bitwise %.4f)" % (nt, info, e_tr, e_last, np.mean(rcv == rcv_r), e_sn, e_g,
                                           np.mean(g == g_r)))
    assert e_tr <= TRACE_TOL and e_last <= TRACE_TOL and e_sn <= TRACE_TOL
    for c in range(3):
        assert K.rel_l2(g[c], g_r[c]) <= GRAD_TOL, "gradient component %d" % c


def test_single_shot_fwi_gradient_vs_reference_solver():
    nt = 600
    wl = W.elastic_single(nt=nt)
    kind, nx, nz, d, dt = wl["kind"], wl["nx"], wl["nz"], wl["d"], wl["dt"]
    sh = wl["shots"][0]
    ref = O.Reference(32)
    par = _par(wl["params"], len(sh["rx"]))
    src2 = wl["src"].reshape(2, nt)
    loc = (np.float32(sh["sx"][0]), np.float32(sh["sz"][0]))
    obs, _ = ref.misfit_grad(kind, par, nx, nz, d, nt, dt, loc, (sh["rx"], sh["rz"]), wl["true"], src2)
    syn_r, g_r = ref.misfit_grad(kind, par, nx, nz, d, nt, dt, loc, (sh["rx"], sh["rz"]), wl["start"], src2, obs)
    w = np.full(nt, dt)
    w[0] = w[-1] = 0.5 * dt
    phi_r = 0.5 * np.sum(w * (syn_r.astype(np.float64) - obs) ** 2)

    P = F.Propagator(0)
    P.set_model(kind, W.convert(kind, wl["start"]), d, d)
    P.set_shots(F.make_params(**wl["params"], tile_shape=-1),
                [F.ShotSpec(0, nx, nt, sh["sx"], sh["sz"], sh["rx"], sh["rz"])])
    g, phi = P.fwi_gradient(W.convert(kind, wl["start"]), [wl["src"]], [obs], seismotype=1)
    P.close()
    e_g = K.rel_l2(g, g_r[:3])
    print("401x801 nt=%d FWI gradient vs the reference solver: %.2e (bitwise %.4f), misfit %.9e vs %.9e" % (
        nt, e_g, np.mean(g == g_r[:3]), phi, phi_r))
    for c in range(3):
        assert K.rel_l2(g[c], g_r[c]) <= GRAD_TOL, "gradient component %d" % c
    assert abs(phi - phi_r) <= 1e-5 * abs(phi_r)


def test_batch_geometry_shots_on_march_units_vs_reference_build():
    kind, nxm, nz, d, dt = O.KIND_ELASTIC, 801, 401, 0.005, 4e-4
    wl = W.elastic_single(nt=8)
    mc = W.convert(kind, wl["start"])
    shots = W.batch_geometry(64, 5001, 2, nxm, d, dt)
    picks = [shots[k] for k in (3, 21, 40, 62)]
    ref = O.Reference(32)
    params = dict(wl["params"])
    specs, srcs, adjs, rcv_r, g_r = [], [], [], [], np.zeros((3, nxm, nz))
    rng = np.random.default_rng(5)
    nts = [s["nt"] // 8 for s in picks]
    params["nt"] = max(nts)
    for s, nt in zip(picks, nts):
        x0, nx = s["x0"], s["nx"]
        ox = np.float32(x0 * d)
        src = _vertical_force(nt, dt)
        par = _par(dict(params, nt=nt), len(s["rx"]))
        mcs = np.ascontiguousarray(mc[:, x0:x0 + nx])
        sl = (np.array(s["sx"], np.float32) - ox, np.array(s["sz"], np.float32))
        rl = (s["rx"] - ox, s["rz"])
        r, full = K.oracle_forward(ref, kind, mcs, src, par, nx, nz, d, sl, rl)
        adj = (rng.standard_normal(r.shape) * np.abs(r).max()).astype(np.float32)
        g_r[:, x0:x0 + nx] += K.oracle_adjoint(ref, kind, mcs, adj, par, nx, nz, d, sl, rl, full)
        del full
        specs.append(F.ShotSpec(x0, nx, nt, s["sx"], s["sz"], s["rx"], s["rz"]))
        srcs.append(src)
        adjs.append(adj)
        rcv_r.append(r)
    P = F.Propagator(0)
    P.set_model(kind, mc, d, d)
    P.set_shots(F.make_params(**params, tile_shape=8), specs)
    rcv = P.forward(srcs, store=True)
    g = P.adjoint(adjs)
    P.close()
    errs = [K.rel_l2(a, b) for a, b in zip(rcv, rcv_r)]
    e_g = K.rel_l2(g, g_r)
    print("batch geometry, shots of %s columns, nt %s, 224x32 marching units: receivers %s, gradient %.2e" % (
        [s["nx"] for s in picks], nts, ["%.1e" % e for e in errs], e_g))
    assert max(errs) <= TRACE_TOL
    for c in range(3):
        assert K.rel_l2(g[c], g_r[c]) <= GRAD_TOL, "gradient component %d" % c


def test_checkpointed_gradient_on_large_grid_crop_vs_reference_build():
    nt, nx, nz, d, dt = 2001, 1001, 301, 0.0025, 2e-4
    kind = O.KIND_ELASTIC
    raw = W.elastic_model(nx, nz, d, seed=0, sigma_cells=20)
    mc = W.convert(kind, W.smoothed(raw, 50))
    src = _vertical_force(nt, dt, 15.0)
    rx = (0.0125 * (1 + np.arange(198))).astype(np.float32)
    rz = np.full(198, 0.01, np.float32)
    sl = (np.array([1.25], np.float32), np.array([0.01], np.float32))
    params = dict(nt=nt, sub=1, dt=dt, bc_top=1, bc_bottom=2, bc_left=2, bc_right=2, taper_top=0, taper_bottom=60,
                  taper_left=60, taper_right=60, taper_strength=0.05)
    ref = O.Reference(32)
    par = _par(params, len(rx))
    rng = np.random.default_rng(9)
    rcv_r, _, adj, g_r = _ref_forward_adjoint(
        ref, kind, mc, src, lambda r: (rng.standard_normal(r.shape) * np.abs(r).max()).astype(np.float32),
        par, nx, nz, d, sl, (rx, rz))
    P = F.Propagator(0)
    P.set_model(kind, mc, d, d)
    P.set_shots(F.make_params(**params, checkpoint_every=200, tile_shape=-1),
                [F.ShotSpec(0, nx, nt, sl[0], sl[1], rx, rz)])
    rcv = P.forward([src], store=True)[0]
    g = P.adjoint([adj])
    info = P.plan_info()
    P.close()
    e_tr, e_g = K.rel_l2(rcv, rcv_r), K.rel_l2(g, g_r)
    print("301x1001 nt=%d, checkpoints every 200 steps (%s): traces %.2e, gradient %.2e (bitwise %.4f)" % (
        nt, info, e_tr, e_g, np.mean(g == g_r)))
    assert e_tr <= TRACE_TOL
    for c in range(3):
        assert K.rel_l2(g[c], g_r[c]) <= GRAD_TOL, "gradient component %d" % c
