"""Oracle loader (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
package.  It binds two CPU implementations of the reference's propagation:

* ``port``      -- oracle/fwi2d_oracle.c, the C restatement (liborc32/64.so);
* ``reference`` -- the reference's own sources compiled by oracle/build_ref.sh
                   (oracle/_ref/libfwi2d_ref32/64.so), present only where the
                   reference tree was available at build time.

Both take the same parameter struct (``Par``) and model/trace layouts as the
reference's ``propagate`` (src/cpp/we_op.cpp:564): model ``[npar][nx][nz]``
already converted, sources ``[ncomp][ns][nt]``, receivers ``[ncomp][nr][nt]``,
snapshots ``[nt/sub+1][ncomp][nx][nz]``, gradient ``[3][nx][nz]``.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

KIND_ELASTIC, KIND_VTI, KIND_ACOUSTIC, KIND_AE = 0, 1, 2, 3


class Par(ctypes.Structure):
    _fields_ = [
        ("nt", ctypes.c_int), ("sub", ctypes.c_int), ("dt", ctypes.c_double),
        ("ns", ctypes.c_int), ("nr", ctypes.c_int),
        ("bc_top", ctypes.c_int), ("bc_bottom", ctypes.c_int), ("bc_left", ctypes.c_int), ("bc_right", ctypes.c_int),
        ("taper_top", ctypes.c_int), ("taper_bottom", ctypes.c_int), ("taper_left", ctypes.c_int), ("taper_right", ctypes.c_int),
        ("taper_strength", ctypes.c_double), ("free_surface_stiffness", ctypes.c_double),
        ("mt", ctypes.c_int),
        ("gdamp_tmin", ctypes.c_double), ("gdamp_tmax", ctypes.c_double), ("gdamp_power", ctypes.c_double),
        ("nza", ctypes.c_int),
        ("water_velocity", ctypes.c_double), ("water_density", ctypes.c_double),
        ("acoustic_source", ctypes.c_int),
    ]


def make_par(**kw):
    d = dict(nt=100, sub=1, dt=4e-4, ns=1, nr=1, bc_top=1, bc_bottom=2, bc_left=2, bc_right=2,
             taper_top=0, taper_bottom=0, taper_left=0, taper_right=0, taper_strength=0.05,
             free_surface_stiffness=1.05, mt=0, gdamp_tmin=0.0, gdamp_tmax=0.0, gdamp_power=1.0,
             nza=0, water_velocity=1.5, water_density=1.0, acoustic_source=1)
    d.update(kw)
    p = Par()
    for k, v in d.items():
        if isinstance(getattr(p, k), float):
            # every real parameter of the reference is data_t: round through float32
            v = float(np.float32(v))
        setattr(p, k, v)
    return p


class Injector(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("ntr", ctypes.c_int),
                ("xind", ctypes.c_void_p), ("zind", ctypes.c_void_p),
                ("xw", ctypes.c_void_p), ("zw", ctypes.c_void_p)]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class _Lib:
    def __init__(self, path, prec, kind):
        self.lib = ctypes.CDLL(path)
        self.prec = prec
        self.kind = kind
        self.dtype = np.float32 if prec == 32 else np.float64

    def arr(self, a):
        return np.ascontiguousarray(a, dtype=self.dtype)

    _resample_symbol = None

    def resample(self, method, adjoint, x, nm, dm, np_, dp, hl=11):
        """The reference's time resampler (operator.cpp:755-856): method
        "sinc" or "linear"; domain axis nm samples at dm, range axis np_ at dp.
        adjoint False: x [ntr][nm] -> [ntr][np_] (interpolation); True:
        x [ntr][np_] -> [ntr][nm] (its adjoint)."""
        f = getattr(self.lib, self._resample_symbol)
        f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                      ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        x = self.arr(x)
        ntr = x.shape[0]
        assert x.shape == (ntr, np_ if adjoint else nm)
        out = np.zeros((ntr, nm if adjoint else np_), self.dtype)
        rc = f(1 if method == "linear" else 0, 1 if adjoint else 0, int(hl), ntr, int(nm), float(dm), int(np_),
               float(dp), _ptr(x), _ptr(out))
        if rc not in (None, 0):
            raise RuntimeError("resampling failed")
        return out


def port_path(prec=32):
    return os.path.join(HERE, "liborc%d.so" % prec)


def reference_path(prec=32):
    return os.path.join(HERE, "_ref", "libfwi2d_ref%d.so" % prec)


def have_reference(prec=32):
    return os.path.exists(reference_path(prec))


def reference_gpu_path():
    return os.path.join(HERE, "_ref", "libfwi2d_ref32_cuda.so")


def have_reference_gpu():
    return os.path.exists(reference_gpu_path())


def reference_b200_path():
    return os.path.join(HERE, "_ref", "libfwi2d_ref32_b200.so")


def have_reference_b200():
    return os.path.exists(reference_b200_path())


class Port(_Lib):
    """The C restatement."""

    def __init__(self, prec=32):
        path = port_path(prec)
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (build with `make -C oracle`)")
        super().__init__(path, prec, "port")
        pre = "orc%d_" % prec
        self._resample_symbol = pre + "resample"
        self._weights = getattr(self.lib, pre + "injector_weights")
        self._prop = getattr(self.lib, pre + "propagate")
        self._conv = getattr(self.lib, pre + "convert_model")
        self._weights.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        self._prop.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Par),
                               ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        self._conv.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]

    def injector_weights(self, itype, lx, lz, nx, nz, dx, dz, ox, oz):
        lx, lz = self.arr(lx), self.arr(lz)
        n = len(lx)
        w = 3 if itype == 0 else 6
        xind = np.zeros((n, 3), np.int32)
        zind = np.zeros((n, 3), np.int32)
        xw = np.zeros((n, 2, w), self.dtype)
        zw = np.zeros((n, 2, w), self.dtype)
        self._weights(itype, n, _ptr(lx), _ptr(lz), nx, nz, dx, dz, ox, oz, _ptr(xind), _ptr(zind), _ptr(xw), _ptr(zw))
        return xind, zind, xw, zw

    def _inj(self, itype, tabs):
        xind, zind, xw, zw = tabs
        j = Injector(itype, len(xind), _ptr(xind), _ptr(zind), _ptr(xw), _ptr(zw))
        j._keep = tabs
        return j

    def convert_model(self, kind, m, forward=True):
        m = self.arr(m).copy()
        self._conv(kind, _ptr(m), m.shape[-1] * m.shape[-2] if m.ndim == 3 else m.size // m.shape[0], 1 if forward else 0)
        return m

    def propagate(self, kind, adj, model, src, rcv, par, nx, nz, dx, dz, ox, oz, inj_locs, ext_locs,
                  inj_type=0, full=None, grad=None, water_inj_locs=None, water_ext_locs=None):
        """Run one shot.  inj_locs / ext_locs: (x array, z array) on the grid
        whose origin is (ox, oz); water locations on the water grid (origin
        (ox, 0)) for the acoustic-elastic propagator."""
        inj = self._inj(inj_type, self.injector_weights(inj_type, inj_locs[0], inj_locs[1], nx, nz, dx, dz, ox, oz)) if inj_locs is not None else None
        ext = self._inj(0, self.injector_weights(0, ext_locs[0], ext_locs[1], nx, nz, dx, dz, ox, oz)) if ext_locs is not None else None
        inja = exta = None
        if kind == KIND_AE:
            nza = par.nza
            wi, we = (water_inj_locs, water_ext_locs)
            if adj:
                wi, we = water_ext_locs, water_inj_locs
            if wi is not None:
                inja = self._inj(0, self.injector_weights(0, wi[0], wi[1], nx, nza, dx, dz, ox, 0.0))
            if we is not None:
                exta = self._inj(0, self.injector_weights(0, we[0], we[1], nx, nza, dx, dz, ox, 0.0))
        rc = self._prop(kind, adj, _ptr(model), _ptr(src), _ptr(rcv),
                        ctypes.byref(inj) if inj else None, ctypes.byref(ext) if ext else None,
                        ctypes.byref(inja) if inja else None, ctypes.byref(exta) if exta else None,
                        _ptr(full), _ptr(grad), ctypes.byref(par), nx, nz, dx, dz)
        if rc != 0:
            raise RuntimeError("oracle propagate failed with status %d" % rc)


class Reference(_Lib):
    """The reference's own sources, compiled by oracle/build_ref.sh."""

    def __init__(self, prec=32):
        path = reference_path(prec)
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (built by oracle/build_ref.sh where the reference is present)")
        super().__init__(path, prec, "reference")
        self._resample_symbol = "ref_resample"
        self._weights = self.lib.ref_injector_weights
        self._weights.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        self._prop = self.lib.ref_propagate
        self._prop.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Par), ctypes.c_int, ctypes.c_int,
                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]

    def injector_weights(self, itype, lx, lz, nx, nz, dx, dz, ox, oz):
        lx, lz = self.arr(lx), self.arr(lz)
        n = len(lx)
        w = 3 if itype == 0 else 6
        xind = np.zeros((n, 3), np.int32)
        zind = np.zeros((n, 3), np.int32)
        xw = np.zeros((n, 2, w), self.dtype)
        zw = np.zeros((n, 2, w), self.dtype)
        self._weights(itype, n, _ptr(lx), _ptr(lz), nx, nz, dx, dz, ox, oz, _ptr(xind), _ptr(zind), _ptr(xw), _ptr(zw))
        return xind, zind, xw, zw

    def convert_model(self, kind, m, forward=True):
        m = self.arr(m).copy()
        f = self.lib.ref_convert_model
        f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        f(kind, _ptr(m), m.shape[-1] * m.shape[-2], 1 if forward else 0)
        return m

    def misfit_grad(self, kind, par, nx, nz, d, nt, dt, src_loc, rcv_locs, model_raw, src, obs=None):
        """The reference operator's forward data (seismotype 1) and, with obs,
        the solver's gradient for residual f(m) - obs (ref_misfit_grad).
        Returns (syn [ncomp][nr][nt], grad or None); ncomp 1 for the
        acoustic propagator, else 2."""
        f = self.lib.ref_misfit_grad
        vp = ctypes.c_void_p
        f.argtypes = [ctypes.c_int, ctypes.POINTER(Par), ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                      ctypes.c_int, ctypes.c_double, self._real(), self._real(), ctypes.c_int, vp, vp, vp, vp, vp, vp, vp]
        rx, rz = self.arr(rcv_locs[0]), self.arr(rcv_locs[1])
        nr = len(rx)
        m = self.arr(model_raw)
        nc = 1 if kind == KIND_ACOUSTIC else 2
        s = self.arr(src).reshape(nc, nt)
        syn = np.zeros((nc, nr, nt), self.dtype)
        o = None if obs is None else self.arr(obs)
        g = None if obs is None else np.zeros(m.shape, self.dtype)
        rc = f(kind, ctypes.byref(par), nx, nz, d, d, nt, dt, src_loc[0], src_loc[1], nr, _ptr(rx), _ptr(rz), _ptr(m),
               _ptr(s), _ptr(o), _ptr(syn), _ptr(g))
        if rc != 0:
            raise RuntimeError("reference misfit/gradient failed")
        return syn, g

    def analyze_model(self, model_raw, nx, nz, dx, dz, data_nt, data_dt, checks):
        """analyzeModel on a copy of the raw model [npar][nx][nz]; checks: the
        16 inputs of ref_analyze_model.  Returns (model, outputs dict)."""
        f = self.lib.ref_analyze_model
        f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                      ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        m = self.arr(model_raw).copy()
        c = np.zeros(20, np.float64)
        c[:16] = checks
        if f(m.shape[0], _ptr(m), nx, nz, dx, dz, data_nt, data_dt, _ptr(c)) != 0:
            raise RuntimeError("reference analyzeModel failed")
        keys = ("courant", "dt", "sub", "nt", "tmax", "vmax", "vmin")
        return m, dict(zip(keys, c[13:20]))

    def bin_write(self, header, vals, axes, datapath):
        """binWrite of vals (axis 1 = last numpy index); axes: (o, d) per axis,
        axis 1 first."""
        f = self.lib.ref_bin_write
        f.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                      ctypes.c_void_p, ctypes.c_char_p]
        v = self.arr(vals)
        n = np.array(v.shape[::-1], np.int32)
        o = np.array([a[0] for a in axes], np.float64)
        d = np.array([a[1] for a in axes], np.float64)
        if f(header.encode(), _ptr(v), len(n), _ptr(n), _ptr(o), _ptr(d), datapath.encode()) != 0:
            raise RuntimeError("reference binWrite failed")

    def bin_read(self, header, ndim0=1, cap=1 << 24):
        """binRead: (array with axis 1 last, [(n, o, d)] of the kept axes)."""
        f = self.lib.ref_bin_read
        f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        out = np.zeros(cap, self.dtype)
        nd = np.zeros(1, np.int32)
        n = np.zeros(6, np.int32)
        o = np.zeros(6, np.float64)
        d = np.zeros(6, np.float64)
        if f(header.encode(), ndim0, _ptr(out), cap, _ptr(nd), _ptr(n), _ptr(o), _ptr(d)) != 0:
            raise RuntimeError("reference binRead failed")
        k = int(nd[0])
        shape = [int(x) for x in n[:k]]
        return out[:int(np.prod(shape))].reshape(shape[::-1]).copy(), [(shape[i], o[i], d[i]) for i in range(k)]

    def dipole_weights(self, x, z, dip, gl, nx, nz, dx, dz, ox=0.0, oz=0.0):
        """dipole_m3 tables: xind, zind [ntr][6], xw, zw [ntr][2][6]."""
        f = self.lib.ref_dipole_weights
        vp = ctypes.c_void_p
        f.argtypes = [ctypes.c_int, vp, vp, vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                      ctypes.c_double, ctypes.c_double, ctypes.c_double, vp, vp, vp, vp]
        x, z, dip = self.arr(x), self.arr(z), self.arr(dip)
        n = len(x)
        xi, zi = np.zeros((n, 6), np.int32), np.zeros((n, 6), np.int32)
        xw, zw = np.zeros((n, 2, 6), self.dtype), np.zeros((n, 2, 6), self.dtype)
        f(n, _ptr(x), _ptr(z), _ptr(dip), gl, nx, nz, dx, dz, ox, oz, _ptr(xi), _ptr(zi), _ptr(xw), _ptr(zw))
        return xi, zi, xw, zw

    def propagate_dipole(self, kind, adj, model, traces, out, par, nx, nz, d, src_loc, rx, rz, rdip, gl, full=None,
                         grad=None):
        """propagate with one delta source and dipole receivers (ref_propagate_dipole)."""
        f = self.lib.ref_propagate_dipole
        vp = ctypes.c_void_p
        f.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp, self._real(), self._real(), ctypes.c_int, vp, vp, vp,
                      ctypes.c_double, vp, vp, ctypes.POINTER(Par), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                      ctypes.c_double]
        rx, rz, rdip = self.arr(rx), self.arr(rz), self.arr(rdip)
        rc = f(kind, adj, _ptr(self.arr(model)), _ptr(self.arr(traces)), _ptr(out), src_loc[0], src_loc[1], len(rx),
               _ptr(rx), _ptr(rz), _ptr(rdip), gl, _ptr(full), _ptr(grad), ctypes.byref(par), nx, nz, d, d)
        if rc != 0:
            raise RuntimeError("reference dipole propagate failed")

    def misfit_grad_rs(self, kind, par, nx, nz, d, nd, dd, prop_dt, method, hl, src_loc, rcv_locs, model_raw, src,
                       obs=None):
        """misfit_grad with sources and data on their own axis (nd samples at
        dd) and the propagation at prop_dt, through the reference's "sinc" or
        "linear" resampler (ref_misfit_grad_rs).  Returns (syn [ncomp][nr][nd],
        grad or None)."""
        f = self.lib.ref_misfit_grad_rs
        vp = ctypes.c_void_p
        f.argtypes = [ctypes.c_int, ctypes.POINTER(Par), ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                      ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                      self._real(), self._real(), ctypes.c_int, vp, vp, vp, vp, vp, vp, vp]
        rx, rz = self.arr(rcv_locs[0]), self.arr(rcv_locs[1])
        nr = len(rx)
        m = self.arr(model_raw)
        nc = 1 if kind == KIND_ACOUSTIC else 2
        s = self.arr(src).reshape(nc, nd)
        syn = np.zeros((nc, nr, nd), self.dtype)
        o = None if obs is None else self.arr(obs)
        g = None if obs is None else np.zeros(m.shape, self.dtype)
        rc = f(kind, ctypes.byref(par), nx, nz, d, d, nd, dd, prop_dt, 1 if method == "linear" else 0, int(hl),
               src_loc[0], src_loc[1], nr, _ptr(rx), _ptr(rz), _ptr(m), _ptr(s), _ptr(o), _ptr(syn), _ptr(g))
        if rc != 0:
            raise RuntimeError("reference misfit/gradient with resampling failed")
        return syn, g

    def misfit_grad_ae(self, par, nx, nz, d, oz, nt, dt, src_loc, rcv_x, rcv_z, rcv_zw, model_raw, src, obs=None,
                       resample=None):
        """Acoustic-elastic forward data [3][nr][nt] (fluid, x, z; seismotype 1)
        and, with obs, the solver's gradient (ref_misfit_grad_ae).  The model
        grid's first row is at depth oz; the fluid layer lies above it.
        resample = (prop_dt, method): nt, dt are then the data axis and the
        propagation runs at prop_dt (ref_misfit_grad_ae_rs)."""
        vp = ctypes.c_void_p
        args = [ctypes.POINTER(Par), ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                ctypes.c_double, ctypes.c_int, ctypes.c_double]
        if resample is None:
            f = self.lib.ref_misfit_grad_ae
            extra = ()
        else:
            f = self.lib.ref_misfit_grad_ae_rs
            args += [ctypes.c_double, ctypes.c_int]
            extra = (float(resample[0]), 1 if resample[1] == "linear" else 0)
        f.argtypes = args + [self._real(), self._real(), ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp]
        rx, rz, rzw = self.arr(rcv_x), self.arr(rcv_z), self.arr(rcv_zw)
        nr = len(rx)
        m = self.arr(model_raw)
        s = self.arr(src)
        syn = np.zeros((3, nr, nt), self.dtype)
        o = None if obs is None else self.arr(obs)
        g = None if obs is None else np.zeros(m.shape, self.dtype)
        rc = f(ctypes.byref(par), nx, nz, d, d, oz, nt, dt, *extra, src_loc[0], src_loc[1], nr, _ptr(rx), _ptr(rz),
               _ptr(rzw), _ptr(m), _ptr(s), _ptr(o), _ptr(syn), _ptr(g))
        if rc != 0:
            raise RuntimeError("reference acoustic-elastic misfit/gradient failed")
        return syn, g

    def fwi_lbfgs(self, kind, par, nx, nz, d, oz, nt, dt, sx, sz, rx, rz, rzw, src, obs, model_raw, niter,
                  ls_a1=0.0):
        """The reference's FWI solver stack (nlls_fwi_eco + lbfgs with the
        regular Wolfe line search, ref_fwi_lbfgs) for niter iterations from
        model_raw [npar][nx][nz].  sx, sz: one source position per shot; rx,
        rz (and rzw, the fluid-layer depths for kind 3): the receivers every
        shot records; src [ncs][ns][nt]; obs [nc][ns * nr][nt].  Returns (the
        final model, the objective function per iteration)."""
        vp = ctypes.c_void_p
        f = self.lib.ref_fwi_lbfgs
        f.argtypes = [ctypes.c_int, ctypes.POINTER(Par), ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                      ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, vp,
                      vp, vp, vp, ctypes.c_int, ctypes.c_double, vp]
        sx, sz, rx, rz = self.arr(sx), self.arr(sz), self.arr(rx), self.arr(rz)
        rzw = self.arr(rz if rzw is None else rzw)
        m = self.arr(model_raw).copy()
        s, o = self.arr(src), self.arr(obs)
        func = np.zeros(niter + 1, self.dtype)
        n = f(kind, ctypes.byref(par), nx, nz, d, d, oz, nt, dt, len(sx), _ptr(sx), _ptr(sz), len(rx), _ptr(rx),
              _ptr(rz), _ptr(rzw), _ptr(s), _ptr(o), _ptr(m), niter, float(ls_a1), _ptr(func))
        if n < 0:
            raise RuntimeError("reference FWI solver run failed")
        return m, func[:n].copy()

    def _real(self):
        return ctypes.c_float if self.dtype == np.float32 else ctypes.c_double

    def propagate(self, kind, adj, model, src, rcv, par, nx, nz, dx, dz, ox, oz, inj_locs, ext_locs,
                  inj_type=0, full=None, grad=None, water_inj_locs=None, water_ext_locs=None):
        def loc(l):
            if l is None:
                return 0, None, None
            x, z = self.arr(l[0]), self.arr(l[1])
            return len(x), x, z
        ni, ix, iz = loc(inj_locs)
        ne, ex, ez = loc(ext_locs)
        nsa, sax, saz = loc(water_inj_locs)
        nra, rax, raz = loc(water_ext_locs)
        rc = self._prop(kind, adj, _ptr(model), _ptr(src), _ptr(rcv), inj_type, ni, _ptr(ix), _ptr(iz),
                        ne, _ptr(ex), _ptr(ez), nsa, _ptr(sax), _ptr(saz), nra, _ptr(rax), _ptr(raz),
                        _ptr(full), _ptr(grad), ctypes.byref(par), nx, nz, dx, dz, ox, oz)
        if rc != 0:
            raise RuntimeError("reference propagate failed with status %d" % rc)


class ReferenceGPU(Reference):
    """The reference's own GPU path (src/cuda, built with -DCUDA into
    oracle/_ref/libfwi2d_ref32_cuda.so by oracle/build_ref.sh): propagate runs
    nl_we_op_e / nl_we_op_vti::propagate_gpu.  For timing the reference's GPU
    implementation only."""

    def __init__(self):
        path = reference_gpu_path()
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (built by oracle/build_ref.sh where the reference is present)")
        _Lib.__init__(self, path, 32, "reference-gpu")
        self._resample_symbol = "ref_resample"
        self._gpu = self.lib.ref_propagate_gpu
        self._gpu.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Par), ctypes.c_int, ctypes.c_int,
                              ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]

    def propagate(self, kind, adj, model, src, rcv, par, nx, nz, dx, dz, ox, oz, inj_locs, ext_locs,
                  inj_type=0, full=None, grad=None, water_inj_locs=None, water_ext_locs=None):
        assert kind in (KIND_ELASTIC, KIND_VTI) and water_inj_locs is None and water_ext_locs is None
        ix, iz = self.arr(inj_locs[0]), self.arr(inj_locs[1])
        ex, ez = self.arr(ext_locs[0]), self.arr(ext_locs[1])
        rc = self._gpu(kind, adj, _ptr(model), _ptr(src), _ptr(rcv), inj_type, len(ix), _ptr(ix), _ptr(iz),
                       len(ex), _ptr(ex), _ptr(ez), _ptr(full), _ptr(grad), ctypes.byref(par), nx, nz, dx, dz, ox, oz)
        if rc != 0:
            raise RuntimeError("reference GPU propagate failed with status %d" % rc)


class ReferenceB200(Reference):
    """The reference built as its maintainer would switch it to fwi2d_b200:
    its own sources with -DCUDA and fwi2d_b200/integration/we_op_b200.cpp as
    the propagate_gpu hook (oracle/_ref/libfwi2d_ref32_b200.so, linked with
    libfwi2d_b200.so).  misfit_grad / misfit_grad_ae run the reference's
    operator classes and solver steps, which call the hook; propagate runs
    the hook directly (ref_propagate_gpu)."""

    def __init__(self):
        path = reference_b200_path()
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (built by oracle/build_ref.sh where the reference is present)")
        _Lib.__init__(self, path, 32, "reference-b200")
        self._resample_symbol = "ref_resample"
        self._gpu = self.lib.ref_propagate_gpu
        self._gpu.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Par), ctypes.c_int, ctypes.c_int,
                              ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]

    def propagate(self, kind, adj, model, src, rcv, par, nx, nz, dx, dz, ox, oz, inj_locs, ext_locs,
                  inj_type=0, full=None, grad=None, water_inj_locs=None, water_ext_locs=None):
        assert kind in (KIND_ELASTIC, KIND_VTI) and water_inj_locs is None and water_ext_locs is None
        ix, iz = self.arr(inj_locs[0]), self.arr(inj_locs[1])
        ex, ez = self.arr(ext_locs[0]), self.arr(ext_locs[1])
        rc = self._gpu(kind, adj, _ptr(model), _ptr(src), _ptr(rcv), inj_type, len(ix), _ptr(ix), _ptr(iz),
                       len(ex), _ptr(ex), _ptr(ez), _ptr(full), _ptr(grad), ctypes.byref(par), nx, nz, dx, dz, ox, oz)
        if rc != 0:
            raise RuntimeError("reference propagate_gpu hook failed with status %d" % rc)
