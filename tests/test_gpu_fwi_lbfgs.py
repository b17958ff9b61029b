"""Acoustic-elastic full-waveform inversion by the reference's own L-BFGS
solver, with every propagation on this library.

The reference's solver stack as main/fwi2d.cpp:234-356 assembles it
(nlls_fwi_eco over nl_we_op_ae, lbfgs with the regular Wolfe line search,
nlsolver.cpp:1207-1345; oracle/ref_shim/ref_driver.cpp ref_fwi_lbfgs) runs
20 iterations on the small acoustic-elastic FWI workload
(fwi2d_b200.workloads.ae_fwi_small: 200 m of water over four elastic layers
and a low-velocity lens, 201 x 61 elastic cells and 21 fluid rows at 10 m,
6 shots, 1201 samples at 1 ms) in two builds of the reference:

* its CPU build (oracle/_ref/libfwi2d_ref32.so), whose run
  tests/golden/make_golden.py stored in tests/golden/fwi_lbfgs_ae_f32.npz;
* the build whose propagate_gpu hook is this library
  (oracle/_ref/libfwi2d_ref32_b200.so with
  fwi2d_b200/integration/we_op_b200.cpp): every objective-function
  evaluation runs the forward and adjoint propagations of the 6 shots on the
  GPU through fwi2d_propagate.

The observed data are modelled again here by the CPU build (the same code
that made the fixture's).  The hook's forward traces are bitwise equal to
the CPU build's on every shot.  The reference sums its FP32 objective
function with an OpenMP reduction whose partial sums follow the thread
count (a different count moved the first misfit by 1.7e-4), so both runs use
8 threads (tests/cases.py set_omp_threads); the order in which the threads'
partial sums combine still varies, at the level of rounding, and two CPU
runs differ by up to 6e-6 of the starting misfit at some iterations.
Checks: the objective function of every iteration agrees with the CPU
run's to 1e-4 of the starting misfit (measured: at most 2e-5), the final
models to 1e-4 relative L2 (the north-star gradient bar; measured 9e-6),
and both runs reduce the misfit by more than half.
"""
import os
import time

import numpy as np
import pytest

import oracle as O
from fwi2d_b200 import workloads as W
from tests import cases as K

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (O.have_reference(32) and O.have_reference_b200()),
                                 reason="reference builds (oracle/_ref) not present")]

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fwi_lbfgs_ae_f32.npz")
TOL = 1e-4


def test_ae_lbfgs_fwi_through_hook_matches_reference_cpu_run():
    g = dict(np.load(GOLD))
    wl = W.ae_fwi_small()
    obs = K.ae_fwi_observed(O.Reference(32), wl)
    assert abs(np.linalg.norm(obs.astype(np.float64)) - float(g["obs_norm"])) <= 1e-6 * float(g["obs_norm"])
    t0 = time.time()
    m, f = K.ae_fwi_lbfgs(O.ReferenceB200(), wl, obs, int(g["niter"]), float(g["ls_a1"]))
    secs = time.time() - t0
    fc, mc = g["func"], g["model"]
    true = wl["true"]
    err = lambda a: np.linalg.norm((a - true).astype(np.float64)) / np.linalg.norm(true.astype(np.float64))
    print("iterations: GPU hook %d, CPU %d (%.1f s through the hook)" % (len(f) - 1, len(fc) - 1, secs))
    for k in range(max(len(f), len(fc))):
        a = f[k] if k < len(f) else float("nan")
        b = fc[k] if k < len(fc) else float("nan")
        print("  iteration %2d: misfit %.7e (hook)  %.7e (CPU)  rel diff %.2e" % (k, a, b, abs(a - b) / fc[0]))
    print("misfit reduction: hook %.4f, CPU %.4f; model error (rel L2 to true) start %.5e, hook %.5e, CPU %.5e; "
          "final models rel L2 %.2e" % (f[-1] / f[0], fc[-1] / fc[0], err(wl["start"]), err(m), err(mc),
                                        K.rel_l2(m, mc)))
    assert len(f) == len(fc)
    assert np.all(np.abs(f - fc) <= TOL * fc[0])
    assert K.rel_l2(m, mc) <= TOL
    assert f[-1] < 0.5 * f[0] and fc[-1] < 0.5 * fc[0]
    assert err(m) < err(wl["start"])
