"""The reference's own classes driving this library through its GPU hook.

oracle/build_ref.sh builds the reference's sources with CUDA defined, as its
maintainer would to switch it to this library, with
fwi2d_b200/integration/we_op_b200.cpp as the propagate_gpu hook (in place of
src/cuda) and libfwi2d_b200.so linked in: oracle/_ref/libfwi2d_ref32_b200.so.
Nothing of the reference is changed; its apply_forward / apply_jacobianT
(src/cpp/we_op.cpp:904-1239) call the hook for every shot.

Checks:
* nl_we_op_e / nl_we_op_vti::propagate_gpu (the hook alone), forward with
  snapshots and adjoint with the imaging condition, against the reference's
  CPU propagate on the same inputs;
* the solver gradient -- the reference's operator forward, residual with
  applyHt, apply_jacobianT with H quadrature and chain rule
  (optimization.hpp:760-890) -- for the elastic, VTI, acoustic and
  acoustic-elastic operators, against the same computed by the reference's
  CPU build (tests/golden/fwi_gradient_*_f32.npz).
Tolerances: the parity bar's 1e-5 (traces) and 1e-4 (gradients); the
measured errors are at or near 0.
"""
import os

import numpy as np
import pytest

import oracle as O
from tests import cases as K

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (O.have_reference(32) and O.have_reference_b200()),
                                 reason="reference builds (oracle/_ref) not present")]

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("kind", [O.KIND_ELASTIC, O.KIND_VTI])
def test_propagate_gpu_hook_matches_reference_cpu(kind):
    nx, nz, d, nt = 96, 72, 0.01, 180
    mc = K.converted(kind, K.model_case(kind, nx, nz, d, seed=31))
    sl, rl = K.geometry(nx, nz, d, nr=18)
    pd = K.par_dict(nt=nt, dt=1e-3)
    src = K.sources(2, nt, 1e-3)
    par = O.make_par(**pd, ns=1, nr=len(rl[0]))
    cpu, hook = O.Reference(32), O.ReferenceB200()
    rcv_c, full_c = K.oracle_forward(cpu, kind, mc, src, par, nx, nz, d, sl, rl)
    rcv_h, full_h = K.oracle_forward(hook, kind, mc, src, par, nx, nz, d, sl, rl)
    adj = np.ascontiguousarray(rcv_c[:, :, ::-1])
    g_c = K.oracle_adjoint(cpu, kind, mc, adj, par, nx, nz, d, sl, rl, full_c)
    g_h = K.oracle_adjoint(hook, kind, mc, adj, par, nx, nz, d, sl, rl, full_c)
    e_tr, e_sn, e_g = K.rel_l2(rcv_h, rcv_c), K.rel_l2(full_h[:nt], full_c[:nt]), K.rel_l2(g_h, g_c)
    print("kind %d through propagate_gpu: traces %.2e (bitwise %.4f), snapshots %.2e, gradient %.2e (bitwise %.4f)" % (
        kind, e_tr, np.mean(rcv_h == rcv_c), e_sn, e_g, np.mean(g_h == g_c)))
    assert e_tr <= 1e-5 and e_sn <= 1e-5
    assert e_g <= 1e-4


@pytest.mark.parametrize("name", ["elastic", "vti", "acoustic"])
def test_solver_gradient_through_hook(name):
    g = dict(np.load(os.path.join(GOLD, "fwi_gradient_%s_f32.npz" % name)))
    kind = int(g["kind"])
    nx, nz, d, nt, dt = int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nt"]), float(g["dt"])
    par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(1, 2, 2, 2), taper=(0, 10, 10, 10)), ns=1, nr=len(g["rx"]))
    hook = O.ReferenceB200()
    geo = ((np.float32(g["sx"]), np.float32(g["sz"])), (g["rx"], g["rz"]))
    syn, grad = hook.misfit_grad(kind, par, nx, nz, d, nt, dt, geo[0], geo[1], g["start"], g["src"], g["obs"])
    w = np.full(nt, dt)
    w[0] = w[-1] = 0.5 * dt
    phi = 0.5 * np.sum(w * (syn.astype(np.float64) - g["obs"]) ** 2)
    npm = 3 if kind != O.KIND_ACOUSTIC else 2
    err = K.rel_l2(grad[:npm], g["grad"][:npm])
    print("%s: the reference solver through propagate_gpu: gradient %.2e (bitwise %.4f), misfit %.9e vs %.9e" % (
        name, err, np.mean(grad[:npm] == g["grad"][:npm]), phi, float(g["misfit"])))
    assert err <= 1e-4
    assert abs(phi - float(g["misfit"])) <= 1e-5 * float(g["misfit"])


def test_acoustic_elastic_solver_gradient_through_hook():
    g = dict(np.load(os.path.join(GOLD, "fwi_gradient_ae_f32.npz")))
    nx, nz, d, nt, dt, nza, oz = (int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nt"]), float(g["dt"]),
                                  int(g["nza"]), float(g["oz"]))
    par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(2, 2, 2, 2), taper=(4, 10, 10, 10)), ns=1, nr=len(g["rx"]),
                     nza=nza, acoustic_source=1)
    hook = O.ReferenceB200()
    syn, grad = hook.misfit_grad_ae(par, nx, nz, d, oz, nt, dt, (np.float32(g["sx"]), np.float32(g["sz"])), g["rx"],
                                    g["rz"], g["rzw"], g["start"], g["src"], g["obs"])
    err = K.rel_l2(grad, g["grad"])
    print("acoustic-elastic: the reference solver through propagate_gpu: gradient %.2e (bitwise %.4f)" % (
        err, np.mean(grad == g["grad"])))
    assert err <= 1e-4
