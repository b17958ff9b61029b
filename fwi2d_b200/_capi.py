"""ctypes binding of include/fwi2d_b200.h (the library's C ABI)."""
import ctypes
import os

import numpy as np

from . import build as _build

ELASTIC, VTI, ACOUSTIC, ACOUSTIC_ELASTIC = 0, 1, 2, 3
SNAP_FP32, SNAP_BF16, SNAP_FP16 = 0, 1, 2
INJ_DELTA, INJ_DDELTA, INJ_DIPOLE = 0, 1, 2

ERR_ARG, ERR_CUDA, ERR_OOM, ERR_STATE, ERR_UNSUPPORTED, ERR_TIMEOUT = -1, -2, -3, -4, -5, -6
ERRORS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "bad state",
          -5: "unsupported", -6: "timeout"}

# every symbol the header declares
SYMBOLS = [
    "fwi2d_last_error", "fwi2d_version", "fwi2d_injector_weights", "fwi2d_ctx_create", "fwi2d_ctx_destroy",
    "fwi2d_set_model", "fwi2d_set_shots", "fwi2d_forward", "fwi2d_adjoint", "fwi2d_upload_traces", "fwi2d_run",
    "fwi2d_sync", "fwi2d_snapshot", "fwi2d_plan_info", "fwi2d_tile_shape_count", "fwi2d_tile_shape",
    "fwi2d_propagate", "fwi2d_update_model", "fwi2d_set_observed", "fwi2d_fwi_gradient", "fwi2d_last_timing",
    "fwi2d_set_stream", "fwi2d_copy_gradient", "fwi2d_set_data_axis", "fwi2d_resample", "fwi2d_propagate_noalloc",
    "fwi2d_noalloc_last_error", "fwi2d_analyze_model", "fwi2d_dipole_weights", "fwi2d_plan_waves",
]

RESAMPLE_SINC, RESAMPLE_LINEAR = 0, 1


class Params(ctypes.Structure):
    _fields_ = [
        ("nt", ctypes.c_int), ("sub", ctypes.c_int), ("dt", ctypes.c_float),
        ("bc_top", ctypes.c_int), ("bc_bottom", ctypes.c_int), ("bc_left", ctypes.c_int), ("bc_right", ctypes.c_int),
        ("taper_top", ctypes.c_int), ("taper_bottom", ctypes.c_int), ("taper_left", ctypes.c_int),
        ("taper_right", ctypes.c_int),
        ("taper_strength", ctypes.c_float), ("free_surface_stiffness", ctypes.c_float),
        ("mt", ctypes.c_int),
        ("gdamp_tmin", ctypes.c_float), ("gdamp_tmax", ctypes.c_float), ("gdamp_power", ctypes.c_float),
        ("nza", ctypes.c_int), ("water_velocity", ctypes.c_float), ("water_density", ctypes.c_float),
        ("acoustic_source", ctypes.c_int),
        ("snapshot_precision", ctypes.c_int), ("checkpoint_every", ctypes.c_int), ("compensated", ctypes.c_int),
        ("tile_shape", ctypes.c_int),
    ]


class ModelCheck(ctypes.Structure):
    _fields_ = [(k, ctypes.c_float) for k in ("vpmin", "vpmax", "vsmin", "vsmax", "rhomin", "rhomax", "deltamin",
                                               "deltamax", "epsilonmin", "epsilonmax")] + [
        ("soft_clip", ctypes.c_int), ("acoustic_elastic", ctypes.c_int), ("water_velocity", ctypes.c_float),
        ("courant", ctypes.c_float), ("dt", ctypes.c_float), ("sub", ctypes.c_int), ("nt", ctypes.c_int),
        ("tmax", ctypes.c_float), ("vmax", ctypes.c_float), ("vmin", ctypes.c_float)]


class Injector(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("ntr", ctypes.c_int),
                ("xind", ctypes.c_void_p), ("zind", ctypes.c_void_p),
                ("xw", ctypes.c_void_p), ("zw", ctypes.c_void_p)]


class Shot(ctypes.Structure):
    _fields_ = [("x0", ctypes.c_int), ("nx", ctypes.c_int), ("nt", ctypes.c_int),
                ("src", Injector), ("rcv", Injector), ("src_water", Injector), ("rcv_water", Injector)]


class Fwi2dError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, msg))
        self.code = code


_lib = None


def lib_path():
    return _build.LIB


def load(build_if_missing=False):
    """Load the in-tree library.  There is no CPU fallback: a missing library
    raises."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path):
        if build_if_missing:
            _build.build()
        else:
            raise FileNotFoundError("libfwi2d_b200.so is not built (python -m fwi2d_b200.build): " + path)
    L = ctypes.CDLL(path)
    vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.fwi2d_last_error.restype = ctypes.c_char_p
    L.fwi2d_injector_weights.argtypes = [i, i, vp, vp, i, i, f, f, f, f, vp, vp, vp, vp]
    L.fwi2d_ctx_create.argtypes = [i, ctypes.POINTER(vp)]
    L.fwi2d_ctx_destroy.argtypes = [vp]
    L.fwi2d_set_model.argtypes = [vp, i, i, i, f, f, vp]
    L.fwi2d_set_shots.argtypes = [vp, ctypes.POINTER(Params), i, ctypes.POINTER(Shot)]
    L.fwi2d_forward.argtypes = [vp, vp, vp, i]
    L.fwi2d_adjoint.argtypes = [vp, vp, vp]
    L.fwi2d_upload_traces.argtypes = [vp, vp, i]
    L.fwi2d_run.argtypes = [vp, i, i]
    L.fwi2d_sync.argtypes = [vp]
    L.fwi2d_snapshot.argtypes = [vp, i, i, vp]
    L.fwi2d_plan_info.argtypes = [vp, vp, vp, vp, vp]
    L.fwi2d_tile_shape.argtypes = [i, vp, vp]
    L.fwi2d_propagate.argtypes = [i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.POINTER(Params), i, i, i, i, f, f]
    L.fwi2d_update_model.argtypes = [vp, vp]
    L.fwi2d_set_observed.argtypes = [vp, vp]
    L.fwi2d_fwi_gradient.argtypes = [vp, vp, vp, vp, i, vp, ctypes.POINTER(ctypes.c_double)]
    L.fwi2d_last_timing.argtypes = [vp, vp, vp]
    L.fwi2d_set_stream.argtypes = [vp, vp]
    L.fwi2d_copy_gradient.argtypes = [vp, vp]
    L.fwi2d_set_data_axis.argtypes = [vp, f, i, i, vp]
    L.fwi2d_resample.argtypes = [i, i, i, i, i, f, i, f, vp, vp]
    L.fwi2d_dipole_weights.argtypes = [i, vp, vp, vp, f, i, i, f, f, f, f, vp, vp, vp, vp]
    L.fwi2d_analyze_model.argtypes = [i, vp, i, i, f, f, i, f, ctypes.POINTER(ModelCheck)]
    L.fwi2d_plan_waves.argtypes = [vp, vp, vp]
    _lib = L
    return L


def check(rc):
    if rc != 0:
        raise Fwi2dError(rc, load().fwi2d_last_error().decode())


def ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)
