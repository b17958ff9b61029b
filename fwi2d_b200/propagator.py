"""Python front end of the C ABI: a batch of shots on one device.

Mirrors the per-shot contract of the reference's ``propagate``
(src/cpp/we_op.cpp:564): the model is already converted (``convert_model``),
traces are ``[ncomp][ntr][nt]`` per shot, gradients are the raw imaging
condition before the H quadrature and the chain rule.
"""
import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _capi as C

PARAM_DEFAULTS = dict(
    nt=0, sub=1, dt=0.0, bc_top=1, bc_bottom=1, bc_left=1, bc_right=1,
    taper_top=0, taper_bottom=0, taper_left=0, taper_right=0, taper_strength=0.05,
    free_surface_stiffness=1.05, mt=0, gdamp_tmin=0.0, gdamp_tmax=0.0, gdamp_power=1.0,
    nza=0, water_velocity=1.5, water_density=1.0, acoustic_source=1,
    snapshot_precision=C.SNAP_FP32, checkpoint_every=0, compensated=0, tile_shape=-1,
)


def make_params(**kw):
    d = dict(PARAM_DEFAULTS)
    unknown = set(kw) - set(d)
    if unknown:
        raise KeyError("unknown parameters: %s" % sorted(unknown))
    d.update(kw)
    p = C.Params()
    for k, v in d.items():
        setattr(p, k, v)
    return p


def injector_tables(itype, locx, locz, nx, nz, dx, dz, ox, oz):
    """delta_m3 / ddelta_m3 tables computed by the library (host side)."""
    L = C.load()
    locx = np.ascontiguousarray(locx, np.float32)
    locz = np.ascontiguousarray(locz, np.float32)
    n = len(locx)
    w = 3 if itype == C.INJ_DELTA else 6
    xind = np.zeros((n, 3), np.int32)
    zind = np.zeros((n, 3), np.int32)
    xw = np.zeros((n, 2, w), np.float32)
    zw = np.zeros((n, 2, w), np.float32)
    C.check(L.fwi2d_injector_weights(itype, n, C.ptr(locx), C.ptr(locz), nx, nz, float(dx), float(dz), float(ox),
                                     float(oz), C.ptr(xind), C.ptr(zind), C.ptr(xw), C.ptr(zw)))
    return xind, zind, xw, zw


def dipole_tables(locx, locz, dip, gl, nx, nz, dx, dz, ox=0.0, oz=0.0):
    """dipole_m3 tables (distributed acoustic sensing receivers, param.gl > 0)
    computed by the library: xind, zind [ntr][6], xw, zw [ntr][2][6]."""
    L = C.load()
    locx, locz, dip = (np.ascontiguousarray(v, np.float32) for v in (locx, locz, dip))
    n = len(locx)
    xind, zind = np.zeros((n, 6), np.int32), np.zeros((n, 6), np.int32)
    xw, zw = np.zeros((n, 2, 6), np.float32), np.zeros((n, 2, 6), np.float32)
    C.check(L.fwi2d_dipole_weights(n, C.ptr(locx), C.ptr(locz), C.ptr(dip), float(gl), nx, nz, float(dx), float(dz),
                                   float(ox), float(oz), C.ptr(xind), C.ptr(zind), C.ptr(xw), C.ptr(zw)))
    return xind, zind, xw, zw


def _injector(itype, tabs):
    if tabs is None:
        return C.Injector(0, 0, None, None, None, None)
    xind, zind, xw, zw = tabs
    return C.Injector(itype, len(xind), C.ptr(xind), C.ptr(zind), C.ptr(xw), C.ptr(zw))


# the reference's param defaults for analyzeModel (src/include/param.hpp:11-46)
MODEL_CHECK_DEFAULTS = dict(vpmin=0.2, vpmax=8.0, vsmin=0.1, vsmax=5.0, rhomin=0.1, rhomax=8.0, deltamin=-0.5,
                            deltamax=1.0, epsilonmin=0.0, epsilonmax=1.0, soft_clip=0, acoustic_elastic=0,
                            water_velocity=1.5, courant=0.6, dt=-1.0, sub=0)


def analyze_model(model_raw, dx, dz, data_nt, data_dt, **par):
    """analyzeModel (src/cpp/we_op.cpp:267-474) through the library's host
    restatement: returns (the clipped raw model [npar][nx][nz], a dict with the
    propagation dt, nt, sub, courant, tmax, vmax, vmin).  par overrides the
    reference's defaults (MODEL_CHECK_DEFAULTS, the `param` field names)."""
    L = C.load()
    m = np.array(model_raw, np.float32, copy=True, order="C")
    npar, nx, nz = m.shape
    kw = dict(MODEL_CHECK_DEFAULTS)
    kw.update(par)
    c = C.ModelCheck(**kw)
    C.check(L.fwi2d_analyze_model(npar, C.ptr(m), nx, nz, float(dx), float(dz), int(data_nt), float(data_dt),
                                  ctypes.byref(c)))
    return m, {k: getattr(c, k) for k in ("dt", "nt", "sub", "courant", "tmax", "vmax", "vmin")}


def prop_nt(nd, dt_data, dt):
    """Propagation length the reference derives for nd data samples at
    dt_data (analyzeModel, src/cpp/we_op.cpp:436-464): tmax = (nd - 1) dt_data in
    single precision, nt = round(tmax / dt) + 1 with dt = min(dt, dt_data)."""
    f = np.float32
    dt = min(f(dt), f(dt_data))
    tmax = f(nd - 1) * f(dt_data)
    return int(math.floor(float(f(tmax / dt)) + 0.5)) + 1   # C round(): halves away from zero


def resample(x, nm, dm, np_, dp, adjoint=False, method="sinc", sinc_half_length=11):
    """The reference's time resampler on the device (sinc_resampler /
    linear_resampler, src/cpp/operator.cpp:760-856): domain axis nm samples at
    dm, range axis np_ samples at dp.  adjoint False: x [ntr][nm] ->
    [ntr][np_]; True: x [ntr][np_] -> [ntr][nm]."""
    L = C.load()
    x = np.ascontiguousarray(x, np.float32)
    ntr = x.shape[0]
    out = np.zeros((ntr, nm if adjoint else np_), np.float32)
    m = C.RESAMPLE_LINEAR if method == "linear" else C.RESAMPLE_SINC
    C.check(L.fwi2d_resample(m, 1 if adjoint else 0, int(sinc_half_length), ntr, int(nm), float(dm), int(np_),
                             float(dp), C.ptr(x), C.ptr(out)))
    return out


@dataclass
class ShotSpec:
    """One shot: its grid is model columns [x0, x0+nx); locations in km
    relative to the model origin (ox, oz).

    Acoustic-elastic propagator (nl_we_op_ae): the fluid layer spans depths
    0 .. oz above the elastic grid (whose first row is at oz); the fluid
    receivers (``water_rcv_*``, as many as the elastic ones) and, with
    ``acoustic_source`` set in the parameters, the source (``water_src_*``)
    are located on the fluid grid, depths from 0."""
    x0: int
    nx: int
    nt: int
    src_x: Sequence[float]
    src_z: Sequence[float]
    rcv_x: Sequence[float]
    rcv_z: Sequence[float]
    mt: bool = False
    water_src_x: Optional[Sequence[float]] = None
    water_src_z: Optional[Sequence[float]] = None
    water_rcv_x: Optional[Sequence[float]] = None
    water_rcv_z: Optional[Sequence[float]] = None


class Propagator:
    """One device context: model, batch plan, forward and adjoint passes."""

    def __init__(self, device=0):
        self.L = C.load()
        h = ctypes.c_void_p()
        C.check(self.L.fwi2d_ctx_create(int(device), ctypes.byref(h)))
        self.h = h
        self.kind = None
        self.nd = None   # per-shot data samples after set_data_axis
        self._keep = []

    def close(self):
        if self.h:
            self.L.fwi2d_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_model(self, kind, model, dx, dz, ox=0.0, oz=0.0):
        m = np.ascontiguousarray(model, np.float32)
        npar, nx, nz = m.shape
        C.check(self.L.fwi2d_set_model(self.h, kind, nx, nz, float(dx), float(dz), C.ptr(m)))
        self.kind, self.nx, self.nz, self.dx, self.dz, self.ox, self.oz = kind, nx, nz, dx, dz, ox, oz

    def set_shots(self, params, shots: List[ShotSpec]):
        self.params = params
        self.shots = shots
        self.nd = None   # a new plan propagates data on its own axis
        arr = (C.Shot * len(shots))()
        keep = []
        self.src_rows, self.rcv_rows = [], []
        ae = self.kind == C.ACOUSTIC_ELASTIC
        fluid_src = ae and bool(params.acoustic_source)
        for i, s in enumerate(shots):
            ox = self.ox + s.x0 * self.dx
            st = C.INJ_DDELTA if s.mt else C.INJ_DELTA
            src = None
            if not fluid_src:
                src = injector_tables(st, s.src_x, s.src_z, s.nx, self.nz, self.dx, self.dz, ox, self.oz)
            rcv = injector_tables(C.INJ_DELTA, s.rcv_x, s.rcv_z, s.nx, self.nz, self.dx, self.dz, ox, self.oz)
            wsrc = wrcv = None
            if ae:
                nza = int(params.nza)
                if fluid_src:
                    wsrc = injector_tables(C.INJ_DELTA, s.water_src_x, s.water_src_z, s.nx, nza, self.dx, self.dz,
                                           ox, 0.0)
                wrcv = injector_tables(C.INJ_DELTA, s.water_rcv_x, s.water_rcv_z, s.nx, nza, self.dx, self.dz, ox,
                                       0.0)
            keep += [src, rcv, wsrc, wrcv]
            arr[i] = C.Shot(s.x0, s.nx, s.nt, _injector(st, src), _injector(C.INJ_DELTA, rcv),
                            _injector(C.INJ_DELTA, wsrc), _injector(C.INJ_DELTA, wrcv))
            nsrc = len(s.water_src_x) if fluid_src else len(s.src_x)
            nc = self.trace_ncomp()
            self.src_rows.append((3 if s.mt else (1 if fluid_src else self.ncomp())) * nsrc)
            self.rcv_rows.append(nc * len(s.rcv_x))
        C.check(self.L.fwi2d_set_shots(self.h, ctypes.byref(params), len(shots), arr))
        self._keep = keep

    def ncomp(self):
        """Wavefield components: 1 (pressure) for the acoustic propagator, else 2."""
        return 1 if self.kind == C.ACOUSTIC else 2

    def trace_ncomp(self):
        """Receiver trace components: the field's, plus the fluid trace first
        for the acoustic-elastic propagator (we_op.cpp:2199-2214)."""
        return 3 if self.kind == C.ACOUSTIC_ELASTIC else self.ncomp()

    def ngrad(self):
        """Gradient components: (K, 1/rho) acoustic, else (lambda, mu, rho)."""
        return 2 if self.kind == C.ACOUSTIC else 3

    # -- host API ---------------------------------------------------------
    def _concat(self, blocks, rows, lengths=None):
        parts = []
        lengths = lengths or [s.nt for s in self.shots]
        for b, r, n in zip(blocks, rows, lengths):
            b = np.asarray(b, np.float32).reshape(r, n)
            parts.append(b.ravel())
        return np.ascontiguousarray(np.concatenate(parts))

    def set_data_axis(self, dt_data, nd, resampling="sinc", sinc_half_length=11):
        """Sources and observed data of fwi_gradient on their own time axis:
        nd[s] samples at dt_data for shot s, resampled to the propagation step
        with the reference's "sinc" or "linear" resampler (param.resampling,
        param.sinc_half_length).  Each shot's nt must be
        prop_nt(nd[s], dt_data, params.dt).  dt_data <= 0 clears it."""
        if dt_data <= 0:
            self.nd = None
            C.check(self.L.fwi2d_set_data_axis(self.h, 0.0, 0, 0, None))
            return
        nd = np.ascontiguousarray(nd, np.int32)
        method = C.RESAMPLE_LINEAR if resampling == "linear" else C.RESAMPLE_SINC
        C.check(self.L.fwi2d_set_data_axis(self.h, float(dt_data), method, int(sinc_half_length), C.ptr(nd)))
        self.nd = [int(v) for v in nd]

    def forward(self, src_blocks, store=True):
        """src_blocks[s]: [ncomp][ntr][nt] traces of shot s.  Returns the
        receiver blocks [ncomp][nr][nt] per shot (ncomp 2, or 1 acoustic)."""
        src = self._concat(src_blocks, self.src_rows)
        out = np.zeros(sum(r * s.nt for r, s in zip(self.rcv_rows, self.shots)), np.float32)
        C.check(self.L.fwi2d_forward(self.h, C.ptr(src), C.ptr(out), 1 if store else 0))
        res, o = [], 0
        for r, s in zip(self.rcv_rows, self.shots):
            nc = self.trace_ncomp()
            res.append(out[o:o + r * s.nt].reshape(nc, r // nc, s.nt))
            o += r * s.nt
        return res

    def adjoint(self, adj_blocks):
        """adj_blocks[s]: [ncomp][nr][nt] adjoint sources of shot s.  Returns
        the raw imaging condition summed over shots: (lambda, mu, rho), or
        (K, 1/rho) for the acoustic propagator."""
        adj = self._concat(adj_blocks, self.rcv_rows)
        g = np.zeros((self.ngrad(), self.nx, self.nz), np.float32)
        C.check(self.L.fwi2d_adjoint(self.h, C.ptr(adj), C.ptr(g)))
        return g

    def snapshot(self, shot, slot):
        s = self.shots[shot]
        out = np.zeros((self.ncomp(), s.nx, self.nz), np.float32)
        C.check(self.L.fwi2d_snapshot(self.h, shot, slot, C.ptr(out)))
        return out

    def update_model(self, model):
        m = np.ascontiguousarray(model, np.float32)
        C.check(self.L.fwi2d_update_model(self.h, C.ptr(m)))

    def set_observed(self, obs_blocks):
        buf = self._concat(obs_blocks, self.rcv_rows, self.nd)
        C.check(self.L.fwi2d_set_observed(self.h, C.ptr(buf)))

    def fwi_gradient(self, model=None, src_blocks=None, obs_blocks=None, seismotype=1, download=True):
        """One device FWI gradient: returns ((vp, vs, rho) gradient -- (vp, rho)
        for the acoustic propagator -- and the misfit), or (None, None) with
        download=False."""
        m = None if model is None else np.ascontiguousarray(model, np.float32)
        src = None if src_blocks is None else self._concat(src_blocks, self.src_rows, self.nd)
        obs = None if obs_blocks is None else self._concat(obs_blocks, self.rcv_rows, self.nd)
        g = np.zeros((self.ngrad(), self.nx, self.nz), np.float32) if download else None
        f = ctypes.c_double(0.0)
        C.check(self.L.fwi2d_fwi_gradient(self.h, C.ptr(m), C.ptr(src), C.ptr(obs), int(seismotype), C.ptr(g),
                                          ctypes.byref(f) if download else None))
        return (g, f.value) if download else (None, None)

    # -- device-resident API ----------------------------------------------
    def upload(self, blocks, adjoint):
        rows = self.rcv_rows if adjoint else self.src_rows
        buf = self._concat(blocks, rows)
        C.check(self.L.fwi2d_upload_traces(self.h, C.ptr(buf), 1 if adjoint else 0))

    def run(self, adjoint, store=True):
        C.check(self.L.fwi2d_run(self.h, 1 if adjoint else 0, 1 if store else 0))

    def sync(self):
        C.check(self.L.fwi2d_sync(self.h))

    def set_stream(self, stream_handle):
        """Order the context's work on a caller stream (an integer cudaStream_t,
        e.g. torch.cuda.current_stream().cuda_stream); 0/None: own stream."""
        C.check(self.L.fwi2d_set_stream(self.h, ctypes.c_void_p(stream_handle) if stream_handle else None))

    def copy_gradient(self, dst_ptr):
        C.check(self.L.fwi2d_copy_gradient(self.h, ctypes.c_void_p(dst_ptr)))

    def last_timing(self):
        f, a = ctypes.c_float(), ctypes.c_float()
        C.check(self.L.fwi2d_last_timing(self.h, ctypes.byref(f), ctypes.byref(a)))
        return f.value, a.value

    def plan_waves(self):
        """(number of waves, snapshot bytes of all shots together)."""
        n, b = ctypes.c_int(), ctypes.c_longlong()
        C.check(self.L.fwi2d_plan_waves(self.h, ctypes.byref(n), ctypes.byref(b)))
        return n.value, b.value

    def plan_info(self):
        lf, la, sh, sb = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int(), ctypes.c_longlong()
        C.check(self.L.fwi2d_plan_info(self.h, ctypes.byref(lf), ctypes.byref(la), ctypes.byref(sh), ctypes.byref(sb)))
        return dict(launches_forward=lf.value, launches_adjoint=la.value, tile_shape=sh.value,
                    snapshot_bytes=sb.value)
