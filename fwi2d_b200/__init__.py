"""fwi2d_b200: B200-native (sm_100a) SBP propagation for nmbader/fwi2d.

The product is libfwi2d_b200.so (C ABI, include/fwi2d_b200.h); this package
binds it.  There is no CPU path: without the built library every call raises.
"""
from ._capi import (ELASTIC, VTI, ACOUSTIC, ACOUSTIC_ELASTIC, SNAP_FP32, SNAP_BF16, SNAP_FP16, INJ_DELTA,
                    INJ_DDELTA, Fwi2dError, load)
from .propagator import (Propagator, ShotSpec, make_params, injector_tables, dipole_tables, prop_nt, resample,
                         analyze_model)

__all__ = ["ELASTIC", "VTI", "ACOUSTIC", "ACOUSTIC_ELASTIC", "SNAP_FP32", "SNAP_BF16", "SNAP_FP16", "INJ_DELTA",
           "INJ_DDELTA", "Fwi2dError", "load", "Propagator", "ShotSpec", "make_params", "injector_tables", "prop_nt",
           "resample", "analyze_model", "dipole_tables"]
