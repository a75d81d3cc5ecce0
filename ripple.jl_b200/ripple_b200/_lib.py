"""ctypes binding of librpl.so (include/rpl.h).

The library is the only compute path: importing this module without the built
library raises immediately, and every call's non-zero status becomes a Python
exception carrying rpl_last_error().
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "librpl.so")

RPL_ABI_VERSION = 2
RPL_OK, RPL_ERR_ARGUMENT, RPL_ERR_DT, RPL_ERR_NONFINITE, RPL_ERR_CUDA, RPL_ERR_OOM, \
    RPL_ERR_STATE, RPL_ERR_UNSUPPORTED, RPL_ERR_DEVICE = range(9)
RPL_FP64, RPL_FP32 = 0, 1
RPL_F64, RPL_F32 = 0, 1
RPL_LAYOUT_XFAST = 0
RPL_STAGE_PREPARE, RPL_STAGE_FINISH, RPL_STAGE_DEFER_SMOOTH = 1, 2, 4
RPL_TRANSPORT_NONE, RPL_TRANSPORT_REFRACTION, RPL_TRANSPORT_INTRINSIC = 0, 1, 2
RPL_DEPTH_INFINITE, RPL_DEPTH_CONSTANT, RPL_DEPTH_FIELD = 0, 1, 2
RPL_WIND_NONE, RPL_WIND_UNIFORM, RPL_WIND_HOLLAND, RPL_WIND_FIELD = 0, 1, 2, 3

_dp = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_d = ctypes.c_double


class RplDesc(ctypes.Structure):
    _fields_ = [
        ("abi_version", _i32), ("precision", _i32), ("transport", _i32), ("device", _i32),
        ("Nx", _i64), ("Ny", _i64), ("Nk", _i64), ("Np", _i64),
        ("dx", _d), ("dy", _d),
        ("xnodes", _dp), ("ynodes", _dp),
        ("periodic_x", _i32), ("periodic_y", _i32),
        ("kappa", _dp), ("kappa_faces", _dp), ("phi", _dp), ("phi_faces", _dp),
        ("depth_kind", _i32), ("depth_constant", _d), ("depth_field", _dp),
        ("gravity", _d), ("memory_limit_bytes", _i64),
        ("xspacings", _dp), ("yspacings", _dp),
    ]


class RplSources(ctypes.Structure):
    _fields_ = [
        ("wind_kind", _i32), ("stress_cap", _i32), ("drag_form", _i32), ("rotation", _i32),
        ("wind_speed", _d), ("wind_direction", _d),
        ("vmax", _d), ("rmax", _d), ("radius", _d), ("shape_parameter", _d),
        ("inflow_angle", _d), ("background_x", _d), ("background_y", _d),
        ("n_track", _i64), ("track_t", _dp), ("track_x", _dp), ("track_y", _dp),
        ("beta_max", _d), ("z_alpha", _d), ("p_in", _d), ("alpha0", _d), ("rho_air", _d),
        ("rho_water", _d), ("von_karman", _d), ("wind_gravity", _d),
        ("has_dissipation", _i32), ("reserved", _i32),
        ("C_ds", _d), ("B_r", _d), ("ds_p", _d), ("sigma_power", _d), ("ds_gravity", _d),
    ]


class RplSourceTerm(ctypes.Structure):
    _fields_ = [("kind", _i32), ("reserved", _i32), ("rate", _d), ("rate_field", _dp), ("direction", _d),
                ("speed", _d), ("speed_field", _dp), ("p", _d * 4), ("gravity", _d)]


class RplEnsembleOptions(ctypes.Structure):
    _fields_ = [("abi_version", _i32), ("use_graph", _i32), ("autotune", _i32), ("direct_cells", _i32),
                ("autotune_cache", ctypes.c_char_p)]


class RplMlpDesc(ctypes.Structure):
    _fields_ = [("abi_version", _i32), ("nbins", _i32), ("hidden", _i32), ("rows", _i32), ("device", _i32),
                ("reserved", _i32), ("seed", ctypes.c_uint64), ("feature_shift", ctypes.c_float),
                ("feature_scale", ctypes.c_float), ("log_floor", ctypes.c_float), ("target_scale", ctypes.c_float)]


class RplError(RuntimeError):
    """A librpl.so call failed; .code is the rpl_status."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class ArgumentError(ValueError):
    """Bad argument (the reference raises Julia's ArgumentError in the same places)."""


_SIGNATURES = {
    "rpl_create": (ctypes.c_int, [ctypes.POINTER(RplDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "rpl_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rpl_set_currents": (ctypes.c_int, [ctypes.c_void_p, _i64, _dp, _i32, _d, _dp, _dp, _dp, _d]),
    "rpl_get_coupling": (ctypes.c_int, [ctypes.c_void_p] + [_dp] * 8),
    "rpl_update_currents": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    "rpl_rows_get": (ctypes.c_int, [ctypes.c_void_p, _i32, _i64, _i64, ctypes.c_void_p]),
    "rpl_rows_set": (ctypes.c_int, [ctypes.c_void_p, _i32, _i64, _i64, ctypes.c_void_p]),
    "rpl_rows_get_on": (ctypes.c_int, [ctypes.c_void_p, _i32, _i64, _i64, ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_rows_set_on": (ctypes.c_int, [ctypes.c_void_p, _i32, _i64, _i64, ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_stage_rows_async": (ctypes.c_int, [ctypes.c_void_p, _d, _i32, _i64, _i64, _i32]),
    "rpl_smooth_rows_async": (ctypes.c_int, [ctypes.c_void_p, _d, _i64, _i64, _i64]),
    "rpl_set_propagation_smoothing": (ctypes.c_int, [ctypes.c_void_p, _i32, _d, _d]),
    "rpl_diagnostics_device": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 5),
    "rpl_snapshot_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, _i32]),
    "rpl_snapshot_wait": (ctypes.c_int, [ctypes.c_void_p]),
    "rpl_host_alloc": (ctypes.c_int, [_i64, ctypes.POINTER(ctypes.c_void_p)]),
    "rpl_host_free": (ctypes.c_int, [ctypes.c_void_p]),
    "rpl_update_currents_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_set_pseudomomentum": (ctypes.c_int, [ctypes.c_void_p, _i64, _dp, _i32, _d, _dp, _d]),
    "rpl_update_coupling": (ctypes.c_int, [ctypes.c_void_p]),
    "rpl_set_sources": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(RplSources)]),
    "rpl_set_wind_field": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    "rpl_set_source_terms": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(RplSourceTerm), _i32]),
    "rpl_set_action": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, _i32, _i32]),
    "rpl_get_action": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, _i32, _i32]),
    "rpl_set_action_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, _i32, _i32]),
    "rpl_get_action_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, _i32, _i32]),
    "rpl_set_clock": (ctypes.c_int, [ctypes.c_void_p, _d, _i64]),
    "rpl_get_clock": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.POINTER(_i64)]),
    "rpl_step": (ctypes.c_int, [ctypes.c_void_p, _d, _i64]),
    "rpl_step_async": (ctypes.c_int, [ctypes.c_void_p, _d, _i64]),
    "rpl_stage_async": (ctypes.c_int, [ctypes.c_void_p, _d, _i32]),
    "rpl_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "rpl_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_tendency": (ctypes.c_int, [ctypes.c_void_p, _dp, _i32]),
    "rpl_diagnostics": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "rpl_device_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_i64)]),
    "rpl_diagnostics_static": (ctypes.c_int, [ctypes.c_void_p, _i32, _i64, _i64, _i64, _i64, ctypes.c_void_p,
                                              _d, _d] + [ctypes.c_void_p] * 6),
    "rpl_ensemble_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), _dp, _i32,
                                           ctypes.POINTER(RplEnsembleOptions), ctypes.POINTER(ctypes.c_void_p)]),
    "rpl_ensemble_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rpl_ensemble_step": (ctypes.c_int, [ctypes.c_void_p, _i64]),
    "rpl_ensemble_step_async": (ctypes.c_int, [ctypes.c_void_p, _i64]),
    "rpl_ensemble_step_sequential_async": (ctypes.c_int, [ctypes.c_void_p, _i64]),
    "rpl_ensemble_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "rpl_ensemble_autotune": (ctypes.c_int, [ctypes.c_void_p, _i32]),
    "rpl_ensemble_shape": (ctypes.c_int, [ctypes.c_void_p, _i32, ctypes.POINTER(_i32), ctypes.POINTER(_i32),
                                          ctypes.POINTER(_i32)]),
    "rpl_ensemble_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_mlp_create": (ctypes.c_int, [ctypes.POINTER(RplMlpDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "rpl_mlp_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rpl_mlp_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_mlp_param_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_i64)]),
    "rpl_mlp_get_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_mlp_set_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_mlp_train_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, _i32, ctypes.c_float, _dp]),
    "rpl_mlp_gradients": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, _i32, ctypes.c_void_p, _dp]),
    "rpl_mlp_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i64, ctypes.c_void_p]),
    "rpl_gemm_bf16": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i32, _i32, _i32,
                                     ctypes.c_void_p]),
    "rpl_gemm_bf16_bounded": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i32, _i32, _i32,
                                             ctypes.c_uint32, ctypes.c_void_p]),
    "rpl_set_learned_gate": (ctypes.c_int, [ctypes.c_void_p, _d]),
    "rpl_learned_fallback_totals": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "rpl_learned_sample": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p]),
    "rpl_set_learned_source": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_learned_outputs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rpl_learned_fallback_cells": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_i64)]),
    "rpl_last_error": (ctypes.c_char_p, []),
    "rpl_abi_version": (ctypes.c_int, []),
}

_lib = None


def load():
    """Load librpl.so once; raise if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"librpl.so not found at {LIB_PATH}; build it with `python build.py` "
                          f"(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.rpl_abi_version() != RPL_ABI_VERSION:
        raise ImportError("librpl.so ABI version mismatch; rebuild it")
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGNATURES)


def check(status):
    if status != RPL_OK:
        msg = load().rpl_last_error().decode("utf-8", "replace")
        if status in (RPL_ERR_ARGUMENT, RPL_ERR_DT):
            raise ArgumentError(msg)
        raise RplError(status, msg)
    return status


def dptr(a):
    """Pointer to a contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.c_contiguous or a.flags.f_contiguous)
    return a.ctypes.data_as(_dp)


def vptr(a):
    return ctypes.c_void_p(a.ctypes.data)
