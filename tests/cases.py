"""Seeded small cases shared by the oracle and the GPU tests.

Units are the reference's: km, s, km/s, g/cm^3.  Each case is a dict with the
converted model, the per-shot geometry and the propagation parameters, sized so
that the oracle finishes in about a second.
"""
import numpy as np

import oracle as O


def ricker(nt, dt, f0, t0):
    t = np.arange(nt) * dt - t0
    a = (np.pi * f0 * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(np.float32)


def smooth_field(rng, nx, nz, sigma):
    from scipy.ndimage import gaussian_filter
    p = gaussian_filter(rng.uniform(-1, 1, (nx, nz)), sigma)
    return p / max(np.abs(p).max(), 1e-12)


def model_case(kind, nx=60, nz=40, d=0.01, seed=0):
    """Raw (unconverted) model: elastic (vp, vs, rho), VTI (+delta, eps), acoustic (vp, rho)."""
    rng = np.random.default_rng(seed)
    z = np.arange(nz) * d
    vp = (2.0 + 0.75 * z)[None, :] * (1 + 0.05 * smooth_field(rng, nx, nz, 3))
    vs = vp / 1.73
    rho = 0.31 * (1000 * vp) ** 0.25
    if kind == O.KIND_ACOUSTIC:
        m = np.stack([vp, rho])
    elif kind == O.KIND_VTI:
        eps = 0.05 + 0.15 * (0.5 + 0.5 * smooth_field(rng, nx, nz, 4))
        dl = 0.10 * (0.5 + 0.5 * smooth_field(rng, nx, nz, 4))
        m = np.stack([vp, vs, rho, dl, eps])
    else:
        m = np.stack([vp, vs, rho])
    return m.astype(np.float32)


def converted(kind, m):
    return O.Port(32).convert_model(kind, m)


def geometry(nx, nz, d, nr=20, sx=None, sz=None, rz=None):
    # off the half-cell position: there the pivot of the discrete delta
    # (std::round of a tie) depends on the working precision
    sx = (0.5 * (nx - 1) + 0.3) * d if sx is None else sx
    sz = 2 * d if sz is None else sz
    rz = 2 * d if rz is None else rz
    rx = np.linspace(3 * d, (nx - 4) * d, nr).astype(np.float32)
    return (np.array([sx], np.float32), np.array([sz], np.float32)), (rx, np.full(nr, rz, np.float32))


def par_dict(nt=200, dt=1e-3, bc=(1, 2, 2, 2), taper=(0, 8, 8, 8), sub=1, mt=0, **kw):
    d = dict(nt=nt, sub=sub, dt=dt, bc_top=bc[0], bc_bottom=bc[1], bc_left=bc[2], bc_right=bc[3],
             taper_top=taper[0], taper_bottom=taper[1], taper_left=taper[2], taper_right=taper[3],
             taper_strength=0.05, mt=mt)
    d.update(kw)
    return d


def sources(ncomp, nt, dt, f0=15.0, t0=0.06, angle=1.3):
    w = ricker(nt, dt, f0, t0)
    if ncomp == 1:
        return w[None, None, :]
    if ncomp == 2:
        return np.stack([w * np.cos(angle), w * np.sin(angle)])[:, None, :].astype(np.float32)
    return np.stack([w * 1.0, w * 0.7, w * 0.4])[:, None, :].astype(np.float32)


def oracle_forward(lib, kind, mc, src, par, nx, nz, d, src_locs, rcv_locs, mt=0):
    nt = par.nt
    nr = len(rcv_locs[0])
    ncomp = 1 if kind == O.KIND_ACOUSTIC else 2
    rcv = np.zeros((ncomp, nr, nt), lib.dtype)
    nslot = 1 + nt // par.sub if par.sub > 0 else 0
    full = np.zeros((nslot, ncomp, nx, nz), lib.dtype) if nslot else None
    lib.propagate(kind, 0, mc.astype(lib.dtype), src.astype(lib.dtype), rcv, par, nx, nz, d, d, 0.0, 0.0,
                  src_locs, rcv_locs, inj_type=1 if mt else 0, full=full)
    return rcv, full


def oracle_adjoint(lib, kind, mc, adj, par, nx, nz, d, src_locs, rcv_locs, full, mt=0):
    ng = 5 if kind == O.KIND_VTI else (2 if kind == O.KIND_ACOUSTIC else 3)
    g = np.zeros((ng, nx, nz), lib.dtype)
    ncs = 1 if kind == O.KIND_ACOUSTIC else (3 if mt else 2)
    srcb = np.zeros((ncs, 1, par.nt), lib.dtype)
    lib.propagate(kind, 1, mc.astype(lib.dtype), adj.astype(lib.dtype), srcb, par, nx, nz, d, d, 0.0, 0.0,
                  rcv_locs, src_locs, inj_type=0, full=full, grad=g)
    return g[:3] if kind != O.KIND_ACOUSTIC else g


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def ae_fwi_par(wl):
    """The reference's param of an acoustic-elastic FWI workload
    (fwi2d_b200.workloads.ae_fwi), for one shot."""
    p = wl["params"]
    keys = ("nt", "sub", "dt", "bc_top", "bc_bottom", "bc_left", "bc_right", "taper_top", "taper_bottom",
            "taper_left", "taper_right", "taper_strength")
    return O.make_par(**{k: p[k] for k in keys}, ns=1, nr=len(wl["rx"]), nza=p["nza"],
                      acoustic_source=p["acoustic_source"])


def ae_fwi_observed(lib, wl):
    """Observed data of an acoustic-elastic FWI workload, modelled shot by shot
    on its true model by the reference's operator (ref_misfit_grad_ae) in the
    layout of its multi-shot range: [3][ns * nr][nt] (fluid, x, z)."""
    par = ae_fwi_par(wl)
    nr, ns, nt = len(wl["rx"]), len(wl["sx"]), wl["nt"]
    obs = np.zeros((3, ns * nr, nt), np.float32)
    for s in range(ns):
        syn, _ = lib.misfit_grad_ae(par, wl["nx"], wl["nz"], wl["d"], wl["oz"], nt, wl["dt"],
                                    (wl["sx"][s], wl["sz"][s]), wl["rx"], wl["rz"], wl["rzw"], wl["true"], wl["src"])
        obs[:, s * nr:(s + 1) * nr] = syn
    return obs


LBFGS_OMP_THREADS = 8


def set_omp_threads(n):
    """Thread count of the OpenMP parallel regions this process starts from
    now on (libgomp's omp_set_num_threads, shared by the reference builds).
    The reference sums its FP32 objective function with an OpenMP reduction
    whose partial sums follow the thread count: runs that compare misfits to
    1e-4 use the same count."""
    import ctypes
    import ctypes.util
    name = ctypes.util.find_library("gomp") or "libgomp.so.1"
    ctypes.CDLL(name).omp_set_num_threads(int(n))


def ae_fwi_lbfgs(lib, wl, obs, niter, ls_a1):
    """The reference's L-BFGS FWI (ref_fwi_lbfgs) of an acoustic-elastic
    workload from its starting model, on LBFGS_OMP_THREADS OpenMP threads;
    returns (final model, misfit per iteration)."""
    ns, nt = len(wl["sx"]), wl["nt"]
    src = np.ascontiguousarray(np.broadcast_to(wl["src"][:, None, :], (1, ns, nt)), np.float32)
    set_omp_threads(LBFGS_OMP_THREADS)
    return lib.fwi_lbfgs(O.KIND_AE, ae_fwi_par(wl), wl["nx"], wl["nz"], wl["d"], wl["oz"], nt, wl["dt"], wl["sx"],
                         wl["sz"], wl["rx"], wl["rz"], wl["rzw"], src, obs, wl["start"], niter, ls_a1)
