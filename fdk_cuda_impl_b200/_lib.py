"""ctypes bindings to libykb.so (the C-ABI of include/ykb.h).

The library is built in-tree (fdk_cuda_impl_b200/libykb.so).  Loading fails
loudly when it is missing: there is no CPU fallback in this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libykb.so")

# ykb_status values; 1..7 are YK::EApiErrorCode
OK = 0
ERR_INVALID_CONFIG = 1
ERR_INVALID_GEOMETRY = 2
ERR_UNSUPPORTED = 3
ERR_INVALID_BUFFER = 5
ERR_STREAMING_STATE = 6
ERR_CUDA = 7
ERR_OUT_OF_MEMORY = 8

PRECISION_FP32 = 0
PRECISION_BF16 = 1
DTYPE_F32 = 0
DTYPE_BF16 = 1

# byte layout of ykb_cone_view == YK::SConeProjGeomVec
VIEW_DTYPE = np.dtype([("src", "<f4", 4), ("detS", "<f4", 4), ("detU", "<f4", 4),
                       ("detV", "<f4", 4), ("angle", "<f4", 4)])


class Volume(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("vox_x", C.c_float), ("vox_y", C.c_float), ("vox_z", C.c_float),
                ("center_x", C.c_float), ("center_y", C.c_float), ("center_z", C.c_float)]


class Filter(C.Structure):
    _fields_ = [("type", C.c_int), ("cutoff", C.c_float), ("gain", C.c_float),
                ("butterworth_order", C.c_float), ("kaiser_beta", C.c_float),
                ("tukey_alpha", C.c_float)]


class CircularFlat(C.Structure):
    _fields_ = [("total_views", C.c_int), ("views_per_turn", C.c_int),
                ("start_angle_rad", C.c_float), ("rotation_direction", C.c_int),
                ("sid_mm", C.c_float), ("sdd_mm", C.c_float), ("z_mm", C.c_float),
                ("source_offset_mm", C.c_float * 3), ("channels", C.c_int), ("rows", C.c_int),
                ("channel_size_mm", C.c_float), ("row_size_mm", C.c_float),
                ("offset_unv_mm", C.c_float * 3), ("tilt_u_rad", C.c_float),
                ("tilt_v_rad", C.c_float), ("tilt_n_rad", C.c_float)]


class YkbError(RuntimeError):
    """A libykb call returned a non-zero ykb_status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"ykb status {code}: {message}")
        self.code = code


# every symbol include/ykb.h declares, with (restype, argtypes)
_P = C.c_void_p
SIGNATURES = {
    "ykb_version": (C.c_int, []),
    "ykb_last_error": (C.c_char_p, []),
    "ykb_regular_scan_range": (C.c_float, [C.c_int, C.c_int]),
    "ykb_build_circular_flat": (C.c_int, [C.POINTER(CircularFlat), _P, C.c_int]),
    "ykb_fdk_plan_create": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_float,
                                      C.POINTER(Volume), C.POINTER(Filter), C.c_int, C.c_int,
                                      C.POINTER(_P)]),
    "ykb_fdk_plan_create_ex": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                         C.c_int, C.POINTER(Volume), C.POINTER(Filter), C.c_int,
                                         C.c_int, C.c_int, C.POINTER(_P)]),
    "ykb_fdk_plan_destroy": (C.c_int, [_P]),
    "ykb_fdk_execute": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, C.c_int, _P]),
    "ykb_fdk_execute_host": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, C.c_int, _P]),
    "ykb_fdk_execute_host_out": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, _P, C.c_int,
                                           _P]),
    "ykb_fdk_filter": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, _P]),
    "ykb_fdk_backproject": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, C.c_int, _P]),
    "ykb_fdk_workspace_bytes": (C.c_size_t, [_P]),
    "ykb_fdk_check": (C.c_int, [_P, _P]),
    "ykb_fdk_test_pipeline_wait": (C.c_int, [_P, C.c_ulonglong, C.c_int]),
    "ykb_fdk_stage_timing": (C.c_int, [_P, C.c_int]),
    "ykb_fdk_stage_times": (C.c_int, [_P, _P, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                      C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "ykb_fdk_filter_static": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(Filter),
                                        _P, C.c_int, _P, _P]),
    "ykb_joseph_plan_create": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.POINTER(Volume),
                                         C.c_int, C.POINTER(_P)]),
    "ykb_joseph_plan_destroy": (C.c_int, [_P]),
    "ykb_joseph_fp": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "ykb_joseph_bp": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "ykb_joseph_workspace_bytes": (C.c_size_t, [_P]),
    "ykb_operator_apply": (C.c_int, [_P, C.c_int, _P, _P, C.c_int, _P]),
    "ykb_joseph_check": (C.c_int, [_P, _P]),
    "ykb_iter_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "ykb_iter_destroy": (C.c_int, [_P]),
    "ykb_dot_f64": (C.c_int, [_P, _P, _P, C.c_size_t, _P, _P]),
    "ykb_cgls_update_xr": (C.c_int, [_P, _P, _P, _P, _P, C.c_size_t, _P, _P, C.c_size_t, _P]),
    "ykb_cgls_update_p": (C.c_int, [_P, _P, _P, _P, _P, C.c_size_t, _P]),
    "ykb_measure_shared_load_gbs": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_double)]),
}

# ykb_task == YK::ETask values
TASK_FP_JOSEPH = 1
TASK_FP_SIDDON = 2
TASK_BP_SIDDON_RAY_DRIVEN = 4
TASK_BP_FDK_PSEUDO_MATCHED = 7
TASK_BP_JOSEPH = 8

_lib = None


def load():
    """Loads libykb.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m fdk_cuda_impl_b200.build` "
                "(this package has no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(code: int) -> None:
    if code != OK:
        msg = load().ykb_last_error()
        raise YkbError(code, msg.decode() if msg else "")


def views_ptr(views: np.ndarray):
    assert views.dtype == VIEW_DTYPE and views.flags["C_CONTIGUOUS"]
    return views.ctypes.data_as(C.c_void_p)
