"""Time resampling on the device: the reference's sinc and linear resamplers
(src/cpp/operator.cpp:755-856) and the FWI gradient with sources and data on
their own time axis (nl_we_op_e::apply_forward / apply_jacobianT,
src/cpp/we_op.cpp:930-1054, 1086-1124, around the propagation).

tests/golden/resample_f32.npz holds the reference's resampler outputs;
tests/golden/fwi_gradient_{elastic,vti,acoustic}_resampled_f32.npz the
reference solver's gradient and misfit for data sampled at 2.5 ms and
propagation at 1 ms (tests/golden/make_golden.py).

* device resampling vs the reference: the weights use the device's double sin
  and cos, which may differ from the host's by an ulp, so the bar is a
  relative max error of 1e-6 (the fraction of bitwise-equal samples is printed);
* the FWI gradient vs the reference solver: relative L2 1e-4, misfit 1e-5;
* a propagation length that does not follow from the data axis is rejected.
"""
import os

import numpy as np
import pytest

import fwi2d_b200 as F
from fwi2d_b200 import workloads as W
from tests import cases as K

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_device_resampler_matches_reference():
    g = dict(np.load(os.path.join(GOLD, "resample_f32.npz")))
    worst, eq, tot = 0.0, 0, 0
    for k, (nm, dm, np_, dp) in enumerate(g["axes"]):
        nm, np_ = int(nm), int(np_)
        for method, hl in (("sinc", 11), ("linear", 11), ("sinc", 4)):
            tag = "%s%d_%d" % (method, hl, k)
            for adjoint, x, ref in ((False, g["x%d" % k], g["fwd_" + tag]), (True, g["y%d" % k], g["adj_" + tag])):
                out = F.resample(x, nm, dm, np_, dp, adjoint=adjoint, method=method, sinc_half_length=hl)
                assert out.shape == ref.shape
                err = float(np.abs(out - ref).max() / np.abs(ref).max())
                worst = max(worst, err)
                eq += int(np.sum(out == ref))
                tot += out.size
                assert err <= 1e-6, (tag, adjoint, err)
    print("resampler: worst relative max error %.2e, bitwise-equal samples %.5f" % (worst, eq / tot))


def _plan(g, method):
    kind = int(g["kind"])
    P = F.Propagator(0)
    P.set_model(kind, W.convert(kind, g["start"]), float(g["d"]), float(g["d"]))
    nt, nd, dd, dt = int(g["nt"]), int(g["nd"]), float(g["dd"]), float(g["dt"])
    assert F.prop_nt(nd, dd, dt) == nt
    shot = F.ShotSpec(0, int(g["nx"]), nt, [float(g["sx"])], [float(g["sz"])], g["rx"], g["rz"])
    params = F.make_params(**K.par_dict(nt=nt, dt=dt, bc=(1, 2, 2, 2), taper=(0, 10, 10, 10)), tile_shape=3)
    P.set_shots(params, [shot])
    P.set_data_axis(dd, [nd], resampling=method)
    return P, kind


@pytest.mark.parametrize("name,method", [("elastic", "sinc"), ("elastic", "linear"), ("vti", "sinc"),
                                         ("acoustic", "linear")])
def test_resampled_fwi_gradient_matches_reference(name, method):
    g = dict(np.load(os.path.join(GOLD, "fwi_gradient_%s_resampled_f32.npz" % name)))
    P, kind = _plan(g, method)
    grad, phi = P.fwi_gradient(W.convert(kind, g["start"]), [g["src"]], [g["obs_" + method]], seismotype=1)
    # a second evaluation on the resident inputs gives the same result
    grad2, phi2 = P.fwi_gradient()
    P.close()
    ref = g["grad_" + method][:grad.shape[0]]
    err = K.rel_l2(grad, ref)
    mis = float(g["misfit_" + method])
    print("%s %s: gradient rel-L2 %.3e (bitwise %.4f)  misfit %.9e vs %.9e" % (
        name, method, err, np.mean(grad == ref), phi, mis))
    assert err <= 1e-4
    assert abs(phi - mis) <= 1e-5 * mis
    assert np.array_equal(grad, grad2) and phi == phi2


def test_data_axis_rejects_inconsistent_length():
    g = dict(np.load(os.path.join(GOLD, "fwi_gradient_elastic_resampled_f32.npz")))
    kind = int(g["kind"])
    P = F.Propagator(0)
    P.set_model(kind, W.convert(kind, g["start"]), float(g["d"]), float(g["d"]))
    nt = int(g["nt"]) - 3
    shot = F.ShotSpec(0, int(g["nx"]), nt, [float(g["sx"])], [float(g["sz"])], g["rx"], g["rz"])
    P.set_shots(F.make_params(**K.par_dict(nt=nt, dt=float(g["dt"]))), [shot])
    with pytest.raises(F.Fwi2dError) as e:
        P.set_data_axis(float(g["dd"]), [int(g["nd"])])
    assert e.value.code == -1 and "round" in str(e.value)
    with pytest.raises(F.Fwi2dError):
        P.set_data_axis(float(g["dt"]) / 2, [2 * int(g["nd"])])   # data step below the propagation step
    P.close()


def test_batched_data_axis_matches_single_shot_plans():
    """Two shots of different record lengths (own nd and nt) in one plan give
    the sum of the gradients and misfits of one-shot plans."""
    g = dict(np.load(os.path.join(GOLD, "fwi_gradient_elastic_resampled_f32.npz")))
    kind, d, dt, dd = int(g["kind"]), float(g["d"]), float(g["dt"]), float(g["dd"])
    nx = int(g["nx"])
    model = W.convert(kind, g["start"])
    nds = [int(g["nd"]), 121]
    nts = [F.prop_nt(n, dd, dt) for n in nds]
    sx = [float(g["sx"]), float(g["sx"]) - 0.2]
    params = F.make_params(**K.par_dict(nt=max(nts), dt=dt, bc=(1, 2, 2, 2), taper=(0, 10, 10, 10)), tile_shape=3)
    shots = [F.ShotSpec(0, nx, nts[k], [sx[k]], [float(g["sz"])], g["rx"], g["rz"]) for k in range(2)]
    srcs = [g["src"][:, :nds[k]] for k in range(2)]
    obs = [g["obs_sinc"][..., :nds[k]] for k in range(2)]

    def run(idx):
        P = F.Propagator(0)
        P.set_model(kind, model, d, d)
        P.set_shots(params, [shots[k] for k in idx])
        P.set_data_axis(dd, [nds[k] for k in idx])
        r = P.fwi_gradient(model, [srcs[k] for k in idx], [obs[k] for k in idx])
        P.close()
        return r
    gb, fb = run([0, 1])
    g0, f0 = run([0])
    g1, f1 = run([1])
    err = K.rel_l2(gb, g0 + g1)
    print("batched data axis: gradient rel-L2 %.3e vs one-shot plans, misfit %.9e vs %.9e" % (err, fb, f0 + f1))
    assert err <= 1e-5
    assert abs(fb - (f0 + f1)) <= 1e-6 * abs(f0 + f1)
