"""Geometry helpers: regular circular flat-panel scans and volume grids.

The per-view geometry is produced by libykb's builder (ykb_build_circular_flat),
which follows the float arithmetic of YKCBCT's buildCircularTrajectory +
buildProjectionGeometry, so views are bit-identical to the reference's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class CircularScan:
    """YK::SRegularCircularScanSpec + YK::SFlatDetectorSpec."""
    total_views: int
    views_per_turn: int
    sid_mm: float
    sdd_mm: float
    channels: int
    rows: int
    channel_size_mm: float
    row_size_mm: float
    start_angle_rad: float = 0.0
    rotation_direction: int = 1
    z_mm: float = 0.0
    source_offset_mm: tuple = (0.0, 0.0, 0.0)
    offset_unv_mm: tuple = (0.0, 0.0, 0.0)
    tilt_rad: tuple = (0.0, 0.0, 0.0)

    def spec(self) -> L.CircularFlat:
        return L.CircularFlat(self.total_views, self.views_per_turn, self.start_angle_rad,
                              self.rotation_direction, self.sid_mm, self.sdd_mm, self.z_mm,
                              (C.c_float * 3)(*self.source_offset_mm), self.channels, self.rows,
                              self.channel_size_mm, self.row_size_mm,
                              (C.c_float * 3)(*self.offset_unv_mm), *self.tilt_rad)

    def views(self) -> np.ndarray:
        out = np.zeros(self.total_views, dtype=L.VIEW_DTYPE)
        spec = self.spec()
        L.check(L.load().ykb_build_circular_flat(C.byref(spec), L.views_ptr(out), len(out)))
        return out

    @property
    def scan_range(self) -> float:
        return float(L.load().ykb_regular_scan_range(self.total_views, self.views_per_turn))


@dataclass
class VolumeGrid:
    """YK::SVolumeGridSpec: voxel centre = center + (i - (n-1)/2) * voxel."""
    nx: int
    ny: int
    nz: int
    voxel_mm: tuple = (1.0, 1.0, 1.0)
    center_mm: tuple = field(default=(0.0, 0.0, 0.0))

    @staticmethod
    def cube(n: int, voxel: float, nz: int | None = None) -> "VolumeGrid":
        return VolumeGrid(n, n, nz or n, (voxel, voxel, voxel))

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    def struct(self) -> L.Volume:
        return L.Volume(self.nx, self.ny, self.nz, *self.voxel_mm, *self.center_mm)


@dataclass
class RampFilter:
    """YK::SAnalyticFilterParams (type = YK::EFdkFilter value)."""
    type: int = 1
    cutoff: float = 0.5
    gain: float = 1.0
    butterworth_order: float = 2.0
    kaiser_beta: float = 8.6
    tukey_alpha: float = 0.5

    NAMES = {"none": 0, "ramlak": 1, "shepplogan": 2, "cosine": 3, "hann": 4, "hamming": 5,
             "blackman": 6, "butterworth": 7, "kaiser": 8, "tukey": 9}

    @staticmethod
    def named(name: str, **kw) -> "RampFilter":
        return RampFilter(RampFilter.NAMES[name.lower().replace("-", "").replace("_", "")], **kw)

    def struct(self) -> L.Filter:
        return L.Filter(self.type, self.cutoff, self.gain, self.butterworth_order,
                        self.kaiser_beta, self.tukey_alpha)
