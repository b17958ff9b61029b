"""The oracle's C restatement against outputs of the reference itself.

tests/golden/*.npz were produced by tests/golden/make_golden.py from the
reference sources compiled in oracle/_ref (FP32 and FP64 builds).  The
restatement must reproduce every sample: model conversion, injector tables,
traces, snapshots and gradients.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from tests import cases as K

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(f for f in glob.glob(os.path.join(GOLD, "*.npz"))
               if not os.path.basename(f).startswith(("fwi_gradient_", "fwi_lbfgs_", "resample_", "analyze_model_",
                                                      "dipole_")))
FWI_FILES = sorted(glob.glob(os.path.join(GOLD, "fwi_gradient_*.npz")))


def test_golden_fixtures_present():
    assert len(FILES) >= 16


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_port_matches_reference(path):
    g = dict(np.load(path))
    prec = 64 if path.endswith("_f64.npz") else 32
    P = O.Port(prec)
    kind = int(g["kind"])
    nx, nz, nt, d = int(g["nx"]), int(g["nz"]), int(g["nt"]), float(g["d"])
    conv_kind = O.KIND_ELASTIC if kind == O.KIND_AE else kind
    mc = P.convert_model(conv_kind, g["raw"])
    assert np.array_equal(mc, g["model"]), "convert_model"
    if kind == O.KIND_AE:
        nza, oz = int(g["nza"]), float(g["oz"])
        par = O.make_par(**K.par_dict(nt=nt, dt=1e-3, bc=(1, 2, 2, 2), taper=(0, 6, 6, 6)), ns=1,
                         nr=len(g["rcv_x"]), nza=nza, acoustic_source=1)
        wsrc = (g["wsrc_x"], g["wsrc_z"])
        rcv = np.zeros_like(g["rcv"])
        full = np.zeros((nt + 1, 2, nx, nz), P.dtype)
        P.propagate(kind, 0, mc, g["src"], rcv, par, nx, nz, d, d, 0.0, oz, None, (g["rcv_x"], g["rcv_ze"]),
                    full=full, water_inj_locs=wsrc, water_ext_locs=(g["rcv_x"], g["rcv_zw"]))
        adj = np.ascontiguousarray(rcv[:, :, ::-1])
        grad = np.zeros_like(g["grad"])
        P.propagate(kind, 1, mc, adj, np.zeros((1, 1, nt), P.dtype), par, nx, nz, d, d, 0.0, oz,
                    (g["rcv_x"], g["rcv_ze"]), None, full=full, grad=grad, water_inj_locs=wsrc,
                    water_ext_locs=(g["rcv_x"], g["rcv_zw"]))
    else:
        mt = int(g["mt"])
        bc = tuple(int(b) for b in g["bc"])
        par = O.make_par(**K.par_dict(nt=nt, dt=1e-3, bc=bc, taper=(0, 6, 6, 6), mt=mt), ns=1, nr=len(g["rcv_x"]))
        sl, rl = (g["src_x"], g["src_z"]), (g["rcv_x"], g["rcv_z"])
        w = P.injector_weights(1 if mt else 0, sl[0], sl[1], nx, nz, d, d, 0.0, 0.0)
        for a, b in zip(w, (g["src_xind"], g["src_zind"], g["src_xw"], g["src_zw"])):
            assert np.array_equal(a, b), "source injector tables"
        w = P.injector_weights(0, rl[0], rl[1], nx, nz, d, d, 0.0, 0.0)
        for a, b in zip(w, (g["rcv_xind"], g["rcv_zind"], g["rcv_xw"], g["rcv_zw"])):
            assert np.array_equal(a, b), "receiver injector tables"
        rcv, full = K.oracle_forward(P, kind, mc, g["src"], par, nx, nz, d, sl, rl, mt=mt)
        adj = np.ascontiguousarray(rcv[:, :, ::-1])
        grad = K.oracle_adjoint(P, kind, mc, adj, par, nx, nz, d, sl, rl, full, mt=mt)
    assert np.array_equal(rcv, g["rcv"]), "traces differ (max %g)" % np.abs(rcv - g["rcv"]).max()
    assert np.array_equal(full[g["snap_idx"]], g["snaps"]), "snapshots"
    assert np.array_equal(grad, g["grad"][:grad.shape[0]]), "gradient"


def test_fp32_vs_fp64_distance_is_small():
    """The FP32 build stays within the FP32 rounding budget of the FP64 oracle
    on these short runs (a sanity bound, not a parity criterion)."""
    a = dict(np.load(os.path.join(GOLD, "elastic_fs_abs_f32.npz")))
    b = dict(np.load(os.path.join(GOLD, "elastic_fs_abs_f64.npz")))
    assert K.rel_l2(a["rcv"], b["rcv"]) < 1e-4
    assert K.rel_l2(a["grad"], b["grad"]) < 1e-3


@pytest.mark.parametrize("path", FWI_FILES, ids=[os.path.basename(f) for f in FWI_FILES])
def test_fwi_gradient_fixture_reproduced_by_reference_build(path):
    """The FWI gradient fixtures (the reference solver's misfit gradient on a
    100 x 80 grid) are reproduced by the reference build in oracle/_ref."""
    if not O.have_reference(32):
        pytest.skip("oracle/_ref is not built")
    g = dict(np.load(path))
    lib = O.Reference(32)
    if "dd" in g and "nza" in g:   # acoustic-elastic, resampled
        nx, nz, d, nd, dd, nza = int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nd"]), float(g["dd"]), int(g["nza"])
        par = O.make_par(**K.par_dict(nt=int(g["nt"]), dt=float(g["dt"]), bc=(2, 2, 2, 2), taper=(4, 10, 10, 10)),
                         ns=1, nr=len(g["rx"]), nza=nza, acoustic_source=1)
        args = (par, nx, nz, d, float(g["oz"]), nd, dd, (g["sx"], g["sz"]), g["rx"], g["rz"], g["rzw"])
        rs = (float(g["dt"]), "sinc")
        syn, _ = lib.misfit_grad_ae(*args, g["true"], g["src"], resample=rs)
        assert np.array_equal(syn, g["obs_sinc"])
        _, grad = lib.misfit_grad_ae(*args, g["start"], g["src"], g["obs_sinc"], resample=rs)
        assert np.array_equal(grad, g["grad_sinc"])
        return
    if "dd" in g:    # data on their own time axis, resampled
        nx, nz, d, nt, dt = int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nt"]), float(g["dt"])
        par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(1, 2, 2, 2), taper=(0, 10, 10, 10)), ns=1, nr=len(g["rx"]))
        geo = ((np.float32(g["sx"]), np.float32(g["sz"])), (g["rx"], g["rz"]))
        for method in [m for m in ("sinc", "linear") if "grad_" + m in g]:
            args = (int(g["kind"]), par, nx, nz, d, int(g["nd"]), float(g["dd"]), dt, method, 11, geo[0], geo[1])
            syn, _ = lib.misfit_grad_rs(*args, g["true"], g["src"])
            assert np.array_equal(syn, g["obs_" + method])
            _, grad = lib.misfit_grad_rs(*args, g["start"], g["src"], g["obs_" + method])
            assert np.array_equal(grad, g["grad_" + method])
        return
    if "nza" in g:   # acoustic-elastic
        nx, nz, d, nt, dt, nza = int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nt"]), float(g["dt"]), int(g["nza"])
        par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(2, 2, 2, 2), taper=(4, 10, 10, 10)), ns=1, nr=len(g["rx"]),
                         nza=nza, acoustic_source=1)
        args = (par, nx, nz, d, float(g["oz"]), nt, dt, (g["sx"], g["sz"]), g["rx"], g["rz"], g["rzw"])
        syn, _ = lib.misfit_grad_ae(*args, g["true"], g["src"])
        assert np.array_equal(syn, g["obs"])
        _, grad = lib.misfit_grad_ae(*args, g["start"], g["src"], g["obs"])
        assert np.array_equal(grad, g["grad"])
        return
    kind, nx, nz, d, nt, dt = int(g["kind"]), int(g["nx"]), int(g["nz"]), float(g["d"]), int(g["nt"]), float(g["dt"])
    par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(1, 2, 2, 2), taper=(0, 10, 10, 10)), ns=1, nr=len(g["rx"]))
    geo = ((np.float32(g["sx"]), np.float32(g["sz"])), (g["rx"], g["rz"]))
    syn, _ = lib.misfit_grad(kind, par, nx, nz, d, nt, dt, geo[0], geo[1], g["true"], g["src"])
    assert np.array_equal(syn, g["obs"])
    _, grad = lib.misfit_grad(kind, par, nx, nz, d, nt, dt, geo[0], geo[1], g["start"], g["src"], g["obs"])
    assert np.array_equal(grad, g["grad"])


def test_resampler_port_matches_reference():
    """The restated sinc and linear resamplers (operator.cpp:760-856) reproduce
    the reference's, forward and adjoint, bit for bit."""
    g = dict(np.load(os.path.join(GOLD, "resample_f32.npz")))
    P = O.Port(32)
    for k, (nm, dm, np_, dp) in enumerate(g["axes"]):
        nm, np_ = int(nm), int(np_)
        for method, hl in (("sinc", 11), ("linear", 11), ("sinc", 4)):
            tag = "%s%d_%d" % (method, hl, k)
            assert np.array_equal(P.resample(method, False, g["x%d" % k], nm, dm, np_, dp, hl), g["fwd_" + tag]), tag
            assert np.array_equal(P.resample(method, True, g["y%d" % k], nm, dm, np_, dp, hl), g["adj_" + tag]), tag


def test_resampler_adjoint_identity():
    """<R x, y> = <x, R^T y> for the restated resamplers (FP64 build)."""
    P = O.Port(64)
    rng = np.random.default_rng(5)
    for method in ("sinc", "linear"):
        x = rng.standard_normal((3, 90))
        y = rng.standard_normal((3, 230))
        a = np.sum(P.resample(method, False, x, 90, 2.5e-3, 230, 9.7e-4) * y)
        b = np.sum(x * P.resample(method, True, y, 90, 2.5e-3, 230, 9.7e-4))
        assert abs(a - b) <= 1e-12 * max(abs(a), 1.0)
