"""ctypes bindings for the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, where it is the checker.  The product package
(fdk_cuda_impl_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

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


class Ellipsoid(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("cx", "cy", "cz", "ax", "ay", "az", "phi", "theta", "psi", "value")]


def build() -> str:
    """Compiles liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        L.orc_regular_scan_range.restype = C.c_float
        L.orc_regular_scan_range.argtypes = [C.c_int, C.c_int]
        for name, args in {
            "orc_build_circular_flat": [C.POINTER(CircularFlat), P],
            "orc_fdk_filter": [P, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(Filter), P, P],
            "orc_fdk_backproject": [P, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(Volume), P, P, C.c_int],
            "orc_fdk": [P, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(Volume), C.POINTER(Filter), P, P, C.c_int],
            "orc_fdk_weighted": [P, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(Volume),
                                 C.POINTER(Filter), P, P, P, C.c_int],
            "orc_fdk_filter_weighted": [P, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(Filter),
                                        P, P, P],
            "orc_parker_weights": [P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, P],
            "orc_fdk_row_band": [P, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(Volume),
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)],
            "orc_fdk_rows": [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                             C.POINTER(Volume), C.POINTER(Filter), P, P, P, C.c_int],
            "orc_fdk_fp32": [P, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(Volume), C.POINTER(Filter), P, P],
            "orc_fdk_derived": [P, C.c_int, C.c_int, C.c_int, C.c_float, P],
            "orc_ramp_kernel": [C.c_int, C.c_double, C.POINTER(Filter), P],
            "orc_joseph_main_axes": [P, C.c_int, C.c_int, C.c_int, P],
            "orc_joseph_fp": [P, C.c_int, C.c_int, C.c_int, C.POINTER(Volume), P, P, C.c_int],
            "orc_joseph_bp": [P, C.c_int, C.c_int, C.c_int, C.POINTER(Volume), P, P],
            "orc_joseph_bp_refweight": [P, C.c_int, C.c_int, C.c_int, C.POINTER(Volume), P, P],
            "orc_pseudo_bp": [P, C.c_int, C.c_int, C.c_int, C.POINTER(Volume), P, P, C.c_int],
            "orc_siddon_fp": [P, C.c_int, C.c_int, C.c_int, C.POINTER(Volume), P, P],
            "orc_siddon_bp": [P, C.c_int, C.c_int, C.c_int, C.POINTER(Volume), P, P],
            "orc_random_ellipsoids": [C.c_uint64, C.c_int, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_double, P],
            "orc_random_spheres": [C.c_uint64, C.c_int, C.c_double, C.c_double, C.c_double,
                                   C.c_double, P],
            "orc_voxelize": [C.POINTER(Volume), P, C.c_int, P],
            "orc_poisson_noise": [P, C.c_size_t, C.c_double, C.c_uint64],
            "orc_uniform": [P, C.c_size_t, C.c_double, C.c_double, C.c_uint64],
            "orc_normal": [P, C.c_size_t, C.c_uint64],
            "orc_mt19937_uniform_pm1": [P, C.c_size_t, C.c_uint32],
        }.items():
            fn = getattr(L, name)
            fn.restype = C.c_int
            fn.argtypes = args
        L.orc_num_threads.restype = C.c_int
        L.orc_set_num_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with code {rc}")


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(n)


def regular_scan_range(total_views: int, views_per_turn: int) -> float:
    return float(lib().orc_regular_scan_range(total_views, views_per_turn))


def volume_struct(shape_zyx, vox, center=(0.0, 0.0, 0.0)) -> Volume:
    nz, ny, nx = shape_zyx
    vx, vy, vz = (vox, vox, vox) if np.isscalar(vox) else vox
    return Volume(nx, ny, nz, vx, vy, vz, *center)


def filter_struct(kind: int = 1, cutoff: float = 0.5, gain: float = 1.0,
                  order: float = 2.0, beta: float = 8.6, alpha: float = 0.5) -> Filter:
    return Filter(kind, cutoff, gain, order, beta, alpha)


def build_circular_flat(total_views, views_per_turn, sid, sdd, channels, rows, du, dv,
                        start_angle=0.0, direction=1, z=0.0, source_offset=(0, 0, 0),
                        offset_unv=(0, 0, 0), tilt=(0, 0, 0)) -> np.ndarray:
    spec = CircularFlat(total_views, views_per_turn, start_angle, direction, sid, sdd, z,
                        (C.c_float * 3)(*source_offset), channels, rows, du, dv,
                        (C.c_float * 3)(*offset_unv), *tilt)
    out = np.zeros(total_views, dtype=VIEW_DTYPE)
    _check(lib().orc_build_circular_flat(C.byref(spec), _ptr(out)), "build geometry")
    return out


def fdk_filter(views, nu, nv, scan_range, filt: Filter, proj) -> np.ndarray:
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    out = np.zeros(proj.shape, dtype=np.float64)
    _check(lib().orc_fdk_filter(_ptr(views), len(views), nu, nv, scan_range, C.byref(filt),
                                _ptr(proj), _ptr(out)), "fdk_filter")
    return out


def fdk_backproject(views, nu, nv, scan_range, vol: Volume, filtered, flags=0) -> np.ndarray:
    filtered = np.ascontiguousarray(filtered, dtype=np.float64)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float64)
    _check(lib().orc_fdk_backproject(_ptr(views), len(views), nu, nv, scan_range, C.byref(vol),
                                     _ptr(filtered), _ptr(out), flags), "fdk_backproject")
    return out


def fdk(views, nu, nv, scan_range, vol: Volume, filt: Filter, proj, flags=0) -> np.ndarray:
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float64)
    _check(lib().orc_fdk(_ptr(views), len(views), nu, nv, scan_range, C.byref(vol),
                         C.byref(filt), _ptr(proj), _ptr(out), flags), "fdk")
    return out


def parker_weights(views, nu, nv, scan_range, start_angle_rad=0.0, direction=1) -> np.ndarray:
    """Parker short-scan weights [n_views][nu] (FP64, range/pi scale included);
    raises when the scan does not qualify (full turn or coverage < pi + 2 fan)."""
    out = np.zeros((len(views), nu), dtype=np.float64)
    _check(lib().orc_parker_weights(_ptr(views), len(views), nu, nv, scan_range,
                                    start_angle_rad, direction, _ptr(out)), "parker_weights")
    return out


def fdk_weighted(views, nu, nv, scan_range, vol: Volume, filt: Filter, proj, row_weights,
                 flags=0) -> np.ndarray:
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    w = None if row_weights is None else np.ascontiguousarray(row_weights, dtype=np.float64)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float64)
    _check(lib().orc_fdk_weighted(_ptr(views), len(views), nu, nv, scan_range, C.byref(vol),
                                  C.byref(filt), _ptr(proj), _ptr(w) if w is not None else None,
                                  _ptr(out), flags), "fdk_weighted")
    return out


def fdk_filter_weighted(views, nu, nv, scan_range, filt: Filter, proj, row_weights) -> np.ndarray:
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    w = np.ascontiguousarray(row_weights, dtype=np.float64)
    out = np.zeros(proj.shape, dtype=np.float64)
    _check(lib().orc_fdk_filter_weighted(_ptr(views), len(views), nu, nv, scan_range,
                                         C.byref(filt), _ptr(proj), _ptr(w), _ptr(out)),
           "fdk_filter_weighted")
    return out


def fdk_row_band(views, nu, nv, scan_range, vol: Volume):
    """(row0, nrows): the detector rows that the volume grid's bilinear
    footprint reads over all views, one row of margin each side."""
    r0, nr = C.c_int(0), C.c_int(0)
    _check(lib().orc_fdk_row_band(_ptr(views), len(views), nu, nv, scan_range, C.byref(vol),
                                  C.byref(r0), C.byref(nr)), "fdk_row_band")
    return r0.value, nr.value


def fdk_rows(views, nu, nv, scan_range, vol: Volume, filt: Filter, proj_rows, row0,
             row_weights=None, flags=0) -> np.ndarray:
    """FDK of a grid whose footprint lies in detector rows [row0, row0 +
    len(proj_rows[0])) of the full nu x nv detector; proj_rows holds only
    those rows.  Equal to fdk() on the full projections for such a grid."""
    proj_rows = np.ascontiguousarray(proj_rows, dtype=np.float32)
    nrows = proj_rows.shape[1]
    w = None if row_weights is None else np.ascontiguousarray(row_weights, dtype=np.float64)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float64)
    _check(lib().orc_fdk_rows(_ptr(views), len(views), nu, nv, row0, nrows, scan_range,
                              C.byref(vol), C.byref(filt), _ptr(proj_rows),
                              _ptr(w) if w is not None else None, _ptr(out), flags), "fdk_rows")
    return out


def fdk_fp32(views, nu, nv, scan_range, vol: Volume, filt: Filter, proj) -> np.ndarray:
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float32)
    _check(lib().orc_fdk_fp32(_ptr(views), len(views), nu, nv, scan_range, C.byref(vol),
                              C.byref(filt), _ptr(proj), _ptr(out)), "fdk_fp32")
    return out


def fdk_derived(views, nu, nv, scan_range) -> np.ndarray:
    out = np.zeros((len(views), 12), dtype=np.float64)
    _check(lib().orc_fdk_derived(_ptr(views), len(views), nu, nv, scan_range, _ptr(out)),
           "fdk_derived")
    return out


def ramp_kernel(nu, du, filt: Filter) -> np.ndarray:
    out = np.zeros(2 * nu - 1, dtype=np.float64)
    _check(lib().orc_ramp_kernel(nu, du, C.byref(filt), _ptr(out)), "ramp_kernel")
    return out


def joseph_main_axes(views, nu, nv) -> np.ndarray:
    out = np.zeros(len(views), dtype=np.int32)
    _check(lib().orc_joseph_main_axes(_ptr(views), len(views), nu, nv, _ptr(out)), "main axes")
    return out


def joseph_fp(views, nu, nv, vol: Volume, volume, flags=0) -> np.ndarray:
    volume = np.ascontiguousarray(volume, dtype=np.float32)
    out = np.zeros((len(views), nv, nu), dtype=np.float64)
    _check(lib().orc_joseph_fp(_ptr(views), len(views), nu, nv, C.byref(vol), _ptr(volume),
                               _ptr(out), flags), "joseph_fp")
    return out


def joseph_bp(views, nu, nv, vol: Volume, proj, reference_weight=False) -> np.ndarray:
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float64)
    fn = lib().orc_joseph_bp_refweight if reference_weight else lib().orc_joseph_bp
    _check(fn(_ptr(views), len(views), nu, nv, C.byref(vol), _ptr(proj), _ptr(out)), "joseph_bp")
    return out


def siddon_fp(views, nu, nv, vol: Volume, volume) -> np.ndarray:
    volume = np.ascontiguousarray(volume, dtype=np.float32)
    out = np.zeros((len(views), nv, nu), dtype=np.float64)
    _check(lib().orc_siddon_fp(_ptr(views), len(views), nu, nv, C.byref(vol), _ptr(volume),
                               _ptr(out)), "siddon_fp")
    return out


def siddon_bp(views, nu, nv, vol: Volume, proj) -> np.ndarray:
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float64)
    _check(lib().orc_siddon_bp(_ptr(views), len(views), nu, nv, C.byref(vol), _ptr(proj),
                               _ptr(out)), "siddon_bp")
    return out


def pseudo_bp(views, nu, nv, vol: Volume, proj, tex=False) -> np.ndarray:
    """BP_FDK_PseudoMatched in FP64 (tex: 8-bit texture interpolation weights)."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float64)
    _check(lib().orc_pseudo_bp(_ptr(views), len(views), nu, nv, C.byref(vol), _ptr(proj),
                               _ptr(out), 1 if tex else 0), "pseudo_bp")
    return out


def random_ellipsoids(seed, count, center_range=25.0, axis_min=3.0, axis_max=25.0,
                      value_min=-0.2, value_max=1.0):
    arr = (Ellipsoid * max(count, 1))()
    _check(lib().orc_random_ellipsoids(seed, count, center_range, axis_min, axis_max,
                                       value_min, value_max, C.cast(arr, C.c_void_p)),
           "random_ellipsoids")
    return [arr[i] for i in range(count)]


def random_spheres(seed, count, center_range=60.0, radius_min=0.5, radius_max=2.0, value=2.0):
    arr = (Ellipsoid * max(count, 1))()
    _check(lib().orc_random_spheres(seed, count, center_range, radius_min, radius_max, value,
                                    C.cast(arr, C.c_void_p)), "random_spheres")
    return [arr[i] for i in range(count)]


def voxelize(vol: Volume, ellipsoids) -> np.ndarray:
    arr = (Ellipsoid * max(len(ellipsoids), 1))(*ellipsoids)
    out = np.zeros((vol.nz, vol.ny, vol.nx), dtype=np.float32)
    _check(lib().orc_voxelize(C.byref(vol), C.cast(arr, C.c_void_p), len(ellipsoids), _ptr(out)),
           "voxelize")
    return out


def poisson_noise(proj: np.ndarray, i0: float, seed: int) -> np.ndarray:
    out = np.ascontiguousarray(proj, dtype=np.float32).copy()
    _check(lib().orc_poisson_noise(_ptr(out), out.size, i0, seed), "poisson_noise")
    return out


def uniform(shape, lo, hi, seed) -> np.ndarray:
    out = np.zeros(shape, dtype=np.float32)
    _check(lib().orc_uniform(_ptr(out), out.size, lo, hi, seed), "uniform")
    return out


def normal(shape, seed) -> np.ndarray:
    out = np.zeros(shape, dtype=np.float32)
    _check(lib().orc_normal(_ptr(out), out.size, seed), "normal")
    return out


def mt19937_uniform_pm1(n: int, seed: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.float32)
    _check(lib().orc_mt19937_uniform_pm1(_ptr(out), n, seed), "mt19937")
    return out
