"""Generate tests/golden/*.npz from the reference itself.

Runs the reference's own propagation code (src/cpp/we_op.cpp et al., compiled
from the reference tree by oracle/build_ref.sh into oracle/_ref/) on small
seeded cases and stores inputs and outputs.  The tests check the oracle's C
restatement and the library's host tables against these files; they never
need the reference tree.

    python tests/golden/make_golden.py [--lbfgs-only]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from tests import cases as K  # noqa: E402


CASES = [
    # name, kind, mt, bc, nx, nz, nt
    ("elastic_fs_abs", O.KIND_ELASTIC, 0, (1, 2, 2, 2), 60, 44, 140),
    ("elastic_all_abs", O.KIND_ELASTIC, 0, (2, 2, 2, 2), 52, 48, 120),
    ("elastic_all_free", O.KIND_ELASTIC, 0, (1, 1, 1, 1), 48, 40, 120),
    ("elastic_mt", O.KIND_ELASTIC, 1, (1, 2, 2, 2), 56, 44, 120),
    ("vti_fs_abs", O.KIND_VTI, 0, (1, 2, 2, 2), 60, 44, 140),
    ("acoustic_dirichlet_abs", O.KIND_ACOUSTIC, 0, (1, 2, 2, 2), 60, 44, 140),
    ("acoustic_neumann", O.KIND_ACOUSTIC, 0, (3, 3, 2, 2), 52, 40, 120),
]


def elastic_like(name, kind, mt, bc, nx, nz, nt, prec):
    d = 0.01
    lib = O.Reference(prec)
    raw = K.model_case(kind, nx, nz, d, seed=11)
    ref_mc = lib.convert_model(kind, raw.astype(lib.dtype))
    sl, rl = K.geometry(nx, nz, d, nr=14)
    ncs = 1 if kind == O.KIND_ACOUSTIC else (3 if mt else 2)
    src = K.sources(ncs, nt, 1e-3).astype(lib.dtype)
    par = O.make_par(**K.par_dict(nt=nt, dt=1e-3, bc=bc, taper=(0, 6, 6, 6), mt=mt), ns=1, nr=14)
    rcv, full = K.oracle_forward(lib, kind, ref_mc, src, par, nx, nz, d, sl, rl, mt=mt)
    adj = np.ascontiguousarray(rcv[:, :, ::-1])
    g = K.oracle_adjoint(lib, kind, ref_mc, adj, par, nx, nz, d, sl, rl, full, mt=mt)
    itype = 1 if mt else 0
    sw = lib.injector_weights(itype, sl[0], sl[1], nx, nz, d, d, 0.0, 0.0)
    rw = lib.injector_weights(0, rl[0], rl[1], nx, nz, d, d, 0.0, 0.0)
    idx = np.linspace(0, nt - 1, 5).astype(int)
    return dict(kind=kind, mt=mt, bc=np.array(bc), nx=nx, nz=nz, nt=nt, d=d, raw=raw, model=ref_mc, src=src,
                src_x=sl[0], src_z=sl[1], rcv_x=rl[0], rcv_z=rl[1], rcv=rcv, snap_idx=idx, snaps=full[idx], grad=g,
                src_xind=sw[0], src_zind=sw[1], src_xw=sw[2], src_zw=sw[3],
                rcv_xind=rw[0], rcv_zind=rw[1], rcv_xw=rw[2], rcv_zw=rw[3])


def ae_case(prec):
    lib = O.Reference(prec)
    nx, nz, d, nt = 56, 40, 0.01, 120
    oz = 0.12
    nza = int(np.floor(oz / d + 1e-6)) + 1
    raw = K.model_case(O.KIND_ELASTIC, nx, nz, d, seed=12)
    raw[0] += 0.5
    raw[1] = raw[0] / 1.8
    mc = lib.convert_model(O.KIND_ELASTIC, raw.astype(lib.dtype))
    par = O.make_par(**K.par_dict(nt=nt, dt=1e-3, bc=(1, 2, 2, 2), taper=(0, 6, 6, 6)), ns=1, nr=14, nza=nza,
                     acoustic_source=1)
    src = K.sources(1, nt, 1e-3, f0=20.0, t0=0.05).astype(lib.dtype)
    rx = np.linspace(0.05, 0.5, 14).astype(np.float32)
    rz_w = np.full(14, 0.06, np.float32)
    rz_e = np.full(14, oz, np.float32)
    wsrc = (np.array([0.3], np.float32), np.array([0.05], np.float32))
    rcv = np.zeros((3, 14, nt), lib.dtype)
    full = np.zeros((nt + 1, 2, nx, nz), lib.dtype)
    lib.propagate(O.KIND_AE, 0, mc, src, rcv, par, nx, nz, d, d, 0.0, oz, None, (rx, rz_e), full=full,
                  water_inj_locs=wsrc, water_ext_locs=(rx, rz_w))
    adj = np.ascontiguousarray(rcv[:, :, ::-1])
    g = np.zeros((3, nx, nz), lib.dtype)
    srcb = np.zeros((1, 1, nt), lib.dtype)
    lib.propagate(O.KIND_AE, 1, mc, adj, srcb, par, nx, nz, d, d, 0.0, oz, (rx, rz_e), None, full=full, grad=g,
                  water_inj_locs=wsrc, water_ext_locs=(rx, rz_w))
    idx = np.linspace(0, nt - 1, 5).astype(int)
    return dict(kind=O.KIND_AE, nx=nx, nz=nz, nt=nt, d=d, oz=oz, nza=nza, raw=raw, model=mc, src=src, rcv_x=rx,
                rcv_zw=rz_w, rcv_ze=rz_e, wsrc_x=wsrc[0], wsrc_z=wsrc[1], rcv=rcv, snap_idx=idx, snaps=full[idx],
                grad=g)


def fwi_case(kind):
    """The solver's gradient through the reference's operator interface
    (nl_we_op_e / nl_we_op_vti / nl_we_op_a forward + apply_jacobianT, residual weighted by
    applyHt), with the finite-difference directional derivative and the
    nonlinear dot-product test (nloper::dotProduct) evaluated on the reference
    itself."""
    lib = O.Reference(32)
    nx, nz, d, nt, dt = 100, 80, 0.01, 400, 1e-3
    rng = np.random.default_rng(1)
    true = K.model_case(kind, nx, nz, d, seed=7)
    start = true.copy()
    from scipy.ndimage import gaussian_filter
    npm = true.shape[0] if kind != O.KIND_VTI else 3   # smoothed parameters: (vp, vs, rho) or (vp, rho)
    for c in range(npm):
        start[c] = gaussian_filter(true[c].astype(np.float64), 4, mode="nearest").astype(np.float32)
    sx, sz = (0.5 * (nx - 1) + 0.3) * d, 0.02
    rx = np.linspace(3 * d, (nx - 4) * d, 30).astype(np.float32)
    rz = np.full(30, 0.02, np.float32)
    nc = 1 if kind == O.KIND_ACOUSTIC else 2
    src = K.sources(nc, nt, dt).reshape(nc, nt)
    dm = np.zeros_like(start)
    for c in range(npm):
        f = gaussian_filter(rng.uniform(-1, 1, (nx, nz)), 5, mode="nearest")
        dm[c] = f / np.abs(f).max() * start[c]
    par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(1, 2, 2, 2), taper=(0, 10, 10, 10)), ns=1, nr=30)
    geo = ((np.float32(sx), np.float32(sz)), (rx, rz))
    obs, _ = lib.misfit_grad(kind, par, nx, nz, d, nt, dt, geo[0], geo[1], true, src)
    w = np.full(nt, dt)
    w[0] = w[-1] = 0.5 * dt

    def phi(m):
        syn, _ = lib.misfit_grad(kind, par, nx, nz, d, nt, dt, geo[0], geo[1], m, src)
        r = syn.astype(np.float64) - obs
        return 0.5 * np.sum(w * r * r)
    syn0, g = lib.misfit_grad(kind, par, nx, nz, d, nt, dt, geo[0], geo[1], start, src, obs)
    eps = 1e-3
    fd = (phi(start + eps * dm) - phi(start - eps * dm)) / (2 * eps)
    an = float(np.sum(g[:npm].astype(np.float64) * dm[:npm]))
    # nloper::dotProduct: residual d for observed data f(m) - d
    rd = rng.uniform(-1, 1, syn0.shape).astype(np.float32) * np.float32(np.abs(syn0).max())
    _, gd = lib.misfit_grad(kind, par, nx, nz, d, nt, dt, geo[0], geo[1], start, src, syn0 - rd)
    sum2 = float(np.sum(gd[:npm].astype(np.float64) * dm[:npm]))
    s1 = []
    for e in (1e-2, 1e-3):
        f1, _ = lib.misfit_grad(kind, par, nx, nz, d, nt, dt, geo[0], geo[1], start + e * dm, src)
        s1.append(float(np.sum(w * rd.astype(np.float64) * (f1.astype(np.float64) - syn0) / e)))
    return dict(kind=kind, nx=nx, nz=nz, d=d, nt=nt, dt=dt, sx=sx, sz=sz, rx=rx, rz=rz, true=true, start=start,
                src=src, obs=obs, dm=dm, grad=g, misfit=phi(start), fd=fd, an=an, dot_residual=rd, dot_sum1=np.array(s1),
                dot_sum2=sum2, grad_dot=gd)


def resample_case():
    """The reference's sinc and linear resamplers (operator.cpp:760-856),
    forward and adjoint, on seeded traces over several axis pairs."""
    lib = O.Reference(32)
    rng = np.random.default_rng(11)
    out = {}
    axes = [(101, 4e-3, 401, 1e-3), (120, 2e-3, 301, 8e-4), (64, 2.5e-3, 170, 9.5e-4), (50, 1e-3, 50, 1e-3),
            (33, 3e-3, 211, 4.7e-4)]
    out["axes"] = np.array([[a[0], a[1], a[2], a[3]] for a in axes], np.float64)
    for k, (nm, dm, np_, dp) in enumerate(axes):
        x = rng.standard_normal((5, nm)).astype(np.float32)
        y = rng.standard_normal((5, np_)).astype(np.float32)
        out["x%d" % k], out["y%d" % k] = x, y
        for method, hl in (("sinc", 11), ("linear", 11), ("sinc", 4)):
            tag = "%s%d_%d" % (method, hl, k)
            out["fwd_" + tag] = lib.resample(method, False, x, nm, dm, np_, dp, hl)
            out["adj_" + tag] = lib.resample(method, True, y, nm, dm, np_, dp, hl)
    return out


def fwi_case_resampled(kind=O.KIND_ELASTIC, methods=("sinc", "linear")):
    """The solver gradient with sources and data sampled at 2.5 ms and the
    propagation at 1 ms: the reference's apply_forward / apply_jacobianT
    resample (sinc, then linear) around the propagation (ref_misfit_grad_rs)."""
    lib = O.Reference(32)
    nx, nz, d, dt, dd, nd = 100, 80, 0.01, 1e-3, 2.5e-3, 161
    true = K.model_case(kind, nx, nz, d, seed=7)
    from scipy.ndimage import gaussian_filter
    start = true.copy()
    for c in range(true.shape[0] if kind != O.KIND_VTI else 3):
        start[c] = gaussian_filter(true[c].astype(np.float64), 4, mode="nearest").astype(np.float32)
    sx, sz = (0.5 * (nx - 1) + 0.3) * d, 0.02
    rx = np.linspace(3 * d, (nx - 4) * d, 30).astype(np.float32)
    rz = np.full(30, 0.02, np.float32)
    nc = 1 if kind == O.KIND_ACOUSTIC else 2
    src = K.sources(nc, nd, dd).reshape(nc, nd)
    nt = 401
    par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(1, 2, 2, 2), taper=(0, 10, 10, 10)), ns=1, nr=30)
    out = dict(kind=kind, nx=nx, nz=nz, d=d, nt=nt, dt=dt, dd=dd, nd=nd, sx=sx, sz=sz, rx=rx, rz=rz, true=true,
               start=start, src=src)
    w = np.full(nd, dd)
    w[0] = w[-1] = 0.5 * dd
    for method in methods:
        geo = ((np.float32(sx), np.float32(sz)), (rx, rz))
        obs, _ = lib.misfit_grad_rs(kind, par, nx, nz, d, nd, dd, dt, method, 11, geo[0], geo[1], true, src)
        syn, g = lib.misfit_grad_rs(kind, par, nx, nz, d, nd, dd, dt, method, 11, geo[0], geo[1], start, src, obs)
        r = syn.astype(np.float64) - obs
        out["obs_" + method], out["syn_" + method], out["grad_" + method] = obs, syn, g
        out["misfit_" + method] = 0.5 * np.sum(w * r * r)
    return out


# analyzeModel inputs: vpmin, vpmax, vsmin, vsmax, rhomin, rhomax, deltamin, deltamax, epsilonmin,
# epsilonmax, soft_clip, acoustic_elastic, water_velocity, courant, dt, sub (param.hpp defaults first)
CHECK_DEFAULTS = [0.2, 8, 0.1, 5, 0.1, 8, -0.5, 1, 0, 1, 0, 0, 1.5, 0.6, -1, 0]
ANALYZE_CASES = [
    # name, kind, overrides (index: value), data_nt, data_dt
    ("elastic_cfl_rounded", O.KIND_ELASTIC, {15: -1}, 1251, 2e-3),
    ("elastic_cfl", O.KIND_ELASTIC, {14: 0}, 1251, 2e-3),
    ("elastic_given_soft", O.KIND_ELASTIC, {14: 4e-4, 10: 1, 15: -1}, 501, 1e-3),
    ("elastic_tight_bounds", O.KIND_ELASTIC, {0: 2.1, 1: 2.6, 3: 1.2, 5: 2.2}, 801, 1.5e-3),
    ("vti", O.KIND_VTI, {7: 0.08, 9: 0.15, 15: -1}, 1001, 2e-3),
    ("acoustic", O.KIND_ACOUSTIC, {0: 2.05, 14: -1}, 1001, 4e-4),
    ("acoustic_elastic", O.KIND_ELASTIC, {11: 1, 12: 1.5, 13: 0.5}, 1201, 2e-3),
    ("data_finer_than_cfl", O.KIND_ELASTIC, {}, 2001, 2e-4),
]


def analyze_case():
    """analyzeModel of the reference (we_op.cpp:267-474) on seeded raw models
    that trip its clips (Vs above Vp/sqrt(2), values outside the bounds, VTI
    delta outside its admissible range) over the dt / sub branches."""
    lib = O.Reference(32)
    out = {}
    nx, nz, d = 40, 30, 0.01
    for k, (name, kind, ov, dnt, ddt) in enumerate(ANALYZE_CASES):
        m = K.model_case(kind, nx, nz, d, seed=20 + k)
        rng = np.random.default_rng(40 + k)
        if kind != O.KIND_ACOUSTIC:
            m[1].flat[rng.integers(0, nx * nz, 30)] *= 1.6          # Vs above Vp/sqrt(2) here and there
        m[0].flat[rng.integers(0, nx * nz, 10)] = 9.0               # above vpmax
        if kind == O.KIND_VTI:
            m[3].flat[rng.integers(0, nx * nz, 20)] = rng.uniform(-0.9, 3.0, 20)   # inadmissible delta
        chk = list(CHECK_DEFAULTS)
        for i, v in ov.items():
            chk[i] = v
        mo, res = lib.analyze_model(m, nx, nz, d, d, dnt, ddt, chk)
        out["name%d" % k] = np.array(name)
        out["in%d" % k] = m.astype(np.float32)
        out["check%d" % k] = np.array(chk, np.float64)
        out["axis%d" % k] = np.array([dnt, ddt], np.float64)
        out["out%d" % k] = mo
        out["res%d" % k] = np.array([res[key] for key in ("courant", "dt", "sub", "nt", "tmax", "vmax", "vmin")])
    out["grid"] = np.array([nx, nz, d])
    return out


def dipole_case():
    """Dipole (DAS) receivers, dipole_m3 (injector.cpp:241-380), on the elastic
    propagator: the reference's tables, its forward traces [2][nr][nt] with
    snapshots, and its adjoint imaging condition for injected traces."""
    lib = O.Reference(32)
    kind, nx, nz, d, nt, gl = O.KIND_ELASTIC, 64, 56, 0.01, 160, 0.03
    mc = K.converted(kind, K.model_case(kind, nx, nz, d, seed=13))
    rng = np.random.default_rng(14)
    nr = 10
    rx = np.linspace(0.08, 0.55, nr).astype(np.float32)
    rz = np.concatenate([np.full(5, 0.013), np.linspace(0.1, 0.45, 5)]).astype(np.float32)
    rdip = rng.uniform(-np.pi, np.pi, nr).astype(np.float32)
    rdip[0], rdip[5] = 0.0, np.float32(np.pi / 2)
    xi, zi, xw, zw = lib.dipole_weights(rx, rz, rdip, gl, nx, nz, d, d)
    sx, sz = np.float32(0.3), np.float32(0.02)
    src = K.sources(2, nt, 1e-3)
    par = O.make_par(**K.par_dict(nt=nt, dt=1e-3), ns=1, nr=nr)
    rcv = np.zeros((2, nr, nt), np.float32)
    full = np.zeros((nt + 1, 2, nx, nz), np.float32)
    lib.propagate_dipole(kind, 0, mc, src, rcv, par, nx, nz, d, (sx, sz), rx, rz, rdip, gl, full=full)
    adj = np.ascontiguousarray(rng.standard_normal((2, nr, nt)).astype(np.float32) * np.abs(rcv).max())
    g = np.zeros((3, nx, nz), np.float32)
    srcb = np.zeros((2, 1, nt), np.float32)
    lib.propagate_dipole(kind, 1, mc, adj, srcb, par, nx, nz, d, (sx, sz), rx, rz, rdip, gl, full=full, grad=g)
    return dict(kind=kind, nx=nx, nz=nz, d=d, nt=nt, gl=gl, model=mc, rx=rx, rz=rz, rdip=rdip, sx=sx, sz=sz, src=src,
                xind=xi, zind=zi, xw=xw, zw=zw, rcv=rcv, adj=adj, grad=g)


SEP_AXES = [(0.0, 0.005), (0.5, 0.005), (0.0, 1.0)]   # (o, d): z, x, parameter


def sep_values():
    return np.random.default_rng(3).standard_normal((3, 20, 16)).astype(np.float32)


def sep_case():
    """A model cube written by the reference's binWrite (IO.hpp:179-222) into
    tests/golden/sep/ (header model_ref.H, binary model_ref.H@, datapath ".")."""
    lib = O.Reference(32)
    d = os.path.join(HERE, "sep")
    os.makedirs(d, exist_ok=True)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        lib.bin_write("model_ref.H", sep_values(), SEP_AXES, ".")
    finally:
        os.chdir(cwd)


def fwi_case_ae():
    """The acoustic-elastic solver gradient (nl_we_op_ae through the
    operator interface, residual weighted by applyHt), fluid source."""
    lib = O.Reference(32)
    nx, nz, d, nt, dt = 90, 60, 0.01, 300, 1e-3
    nza = 16
    oz = (nza - 1) * d
    true = K.model_case(O.KIND_ELASTIC, nx, nz, d, seed=17)
    true[0] += 0.5
    true[1] = true[0] / 1.8
    start = true.copy()
    from scipy.ndimage import gaussian_filter
    for c in range(3):
        start[c] = gaussian_filter(true[c].astype(np.float64), 4, mode="nearest").astype(np.float32)
    sx, sz = np.float32(0.41 * nx * d), np.float32(0.05)
    rx = np.linspace(3 * d, (nx - 4) * d, 24).astype(np.float32)
    rz = np.full(24, oz + 0.02, np.float32)
    rzw = np.full(24, 0.03, np.float32)
    src = K.sources(1, nt, dt, f0=15.0).reshape(1, nt)
    par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(2, 2, 2, 2), taper=(4, 10, 10, 10)), ns=1, nr=24, nza=nza,
                     acoustic_source=1)
    obs, _ = lib.misfit_grad_ae(par, nx, nz, d, oz, nt, dt, (sx, sz), rx, rz, rzw, true, src)
    syn0, g = lib.misfit_grad_ae(par, nx, nz, d, oz, nt, dt, (sx, sz), rx, rz, rzw, start, src, obs)
    w = np.full(nt, dt)
    w[0] = w[-1] = 0.5 * dt
    r = syn0.astype(np.float64) - obs
    return dict(nx=nx, nz=nz, d=d, nt=nt, dt=dt, nza=nza, oz=oz, sx=sx, sz=sz, rx=rx, rz=rz, rzw=rzw, true=true,
                start=start, src=src, obs=obs, grad=g, misfit=0.5 * np.sum(w * r * r))


def fwi_case_ae_resampled():
    """fwi_case_ae with the source and data sampled at 2.5 ms, the propagation
    at 1 ms and the sinc resampler (ref_misfit_grad_ae_rs)."""
    lib = O.Reference(32)
    nx, nz, d, dt, dd, nd = 90, 60, 0.01, 1e-3, 2.5e-3, 121
    nt = 301
    nza = 16
    oz = (nza - 1) * d
    true = K.model_case(O.KIND_ELASTIC, nx, nz, d, seed=17)
    true[0] += 0.5
    true[1] = true[0] / 1.8
    start = true.copy()
    from scipy.ndimage import gaussian_filter
    for c in range(3):
        start[c] = gaussian_filter(true[c].astype(np.float64), 4, mode="nearest").astype(np.float32)
    sx, sz = np.float32(0.41 * nx * d), np.float32(0.05)
    rx = np.linspace(3 * d, (nx - 4) * d, 24).astype(np.float32)
    rz = np.full(24, oz + 0.02, np.float32)
    rzw = np.full(24, 0.03, np.float32)
    src = K.sources(1, nd, dd, f0=15.0).reshape(1, nd)
    par = O.make_par(**K.par_dict(nt=nt, dt=dt, bc=(2, 2, 2, 2), taper=(4, 10, 10, 10)), ns=1, nr=24, nza=nza,
                     acoustic_source=1)
    rs = (dt, "sinc")
    obs, _ = lib.misfit_grad_ae(par, nx, nz, d, oz, nd, dd, (sx, sz), rx, rz, rzw, true, src, resample=rs)
    syn0, g = lib.misfit_grad_ae(par, nx, nz, d, oz, nd, dd, (sx, sz), rx, rz, rzw, start, src, obs, resample=rs)
    w = np.full(nd, dd)
    w[0] = w[-1] = 0.5 * dd
    r = syn0.astype(np.float64) - obs
    return dict(nx=nx, nz=nz, d=d, nt=nt, dt=dt, dd=dd, nd=nd, nza=nza, oz=oz, sx=sx, sz=sz, rx=rx, rz=rz, rzw=rzw,
                true=true, start=start, src=src, obs_sinc=obs, grad_sinc=g, misfit_sinc=0.5 * np.sum(w * r * r))


LBFGS_ITERS, LBFGS_A1 = 20, 0.01


def fwi_lbfgs_ae_case():
    """The reference's L-BFGS FWI (main/fwi2d.cpp's solver stack through
    ref_fwi_lbfgs) on the small acoustic-elastic FWI workload, 20 iterations,
    initial step 1 % of the model norm: the objective function per iteration
    and the final model.  The observed data are not stored: the tests model
    them again with the reference build (tests/cases.py ae_fwi_observed)."""
    from fwi2d_b200 import workloads as W
    lib = O.Reference(32)
    wl = W.ae_fwi_small()
    obs = K.ae_fwi_observed(lib, wl)
    m, f = K.ae_fwi_lbfgs(lib, wl, obs, LBFGS_ITERS, LBFGS_A1)
    return dict(niter=LBFGS_ITERS, ls_a1=LBFGS_A1, func=f, model=m, obs_norm=np.linalg.norm(obs.astype(np.float64)))


def main():
    if not O.have_reference(32):
        sys.exit("oracle/_ref is not built (oracle/build_ref.sh needs the reference tree)")
    if "--lbfgs-only" in sys.argv:   # the solver run alone takes minutes
        np.savez_compressed(os.path.join(HERE, "fwi_lbfgs_ae_f32.npz"), **fwi_lbfgs_ae_case())
        return
    for prec in (32, 64):
        for name, kind, mt, bc, nx, nz, nt in CASES:
            out = elastic_like(name, kind, mt, bc, nx, nz, nt, prec)
            np.savez_compressed(os.path.join(HERE, "%s_f%d.npz" % (name, prec)), **out)
        np.savez_compressed(os.path.join(HERE, "acoustic_elastic_f%d.npz" % prec), **ae_case(prec))
    for kind, name in ((O.KIND_ELASTIC, "elastic"), (O.KIND_VTI, "vti"), (O.KIND_ACOUSTIC, "acoustic")):
        np.savez_compressed(os.path.join(HERE, "fwi_gradient_%s_f32.npz" % name), **fwi_case(kind))
    np.savez_compressed(os.path.join(HERE, "fwi_gradient_ae_f32.npz"), **fwi_case_ae())
    np.savez_compressed(os.path.join(HERE, "fwi_gradient_ae_resampled_f32.npz"), **fwi_case_ae_resampled())
    np.savez_compressed(os.path.join(HERE, "resample_f32.npz"), **resample_case())
    np.savez_compressed(os.path.join(HERE, "analyze_model_f32.npz"), **analyze_case())
    sep_case()
    np.savez_compressed(os.path.join(HERE, "dipole_f32.npz"), **dipole_case())
    np.savez_compressed(os.path.join(HERE, "fwi_gradient_elastic_resampled_f32.npz"), **fwi_case_resampled())
    np.savez_compressed(os.path.join(HERE, "fwi_gradient_vti_resampled_f32.npz"),
                        **fwi_case_resampled(O.KIND_VTI, ("sinc",)))
    np.savez_compressed(os.path.join(HERE, "fwi_gradient_acoustic_resampled_f32.npz"),
                        **fwi_case_resampled(O.KIND_ACOUSTIC, ("linear",)))
    np.savez_compressed(os.path.join(HERE, "fwi_lbfgs_ae_f32.npz"), **fwi_lbfgs_ae_case())
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
