"""Seeded synthetic cases shared by the tests and the benchmark.

Inputs are generated with the oracle's seeded generators (mt19937_64 based)
so the CUDA path and the oracle see identical arrays.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from fdk_cuda_impl_b200.geometry import CircularScan, RampFilter, VolumeGrid


@dataclass
class Case:
    name: str
    scan: CircularScan
    grid: VolumeGrid
    filt: RampFilter
    n_ellipsoids: int = 10
    seed: int = 1
    noise_i0: float | None = None
    center_range: float = 25.0
    axis_min: float = 3.0
    axis_max: float = 25.0


def c1(views=180, n=128, nu=192, nv=128):
    """Plain FP32 FDK case (128^3 @ 0.5 mm, 180 views, 192x128 @ 0.8 mm, 500/1000 mm)."""
    return Case("c1", CircularScan(views, views, 500.0, 1000.0, nu, nv, 0.8, 0.8),
                VolumeGrid.cube(n, 0.5), RampFilter.named("ramlak"))


def c1_small():
    """C1 geometry reduced so the FP64 oracle finishes in about a second."""
    return Case("c1-small", CircularScan(60, 60, 500.0, 1000.0, 96, 64, 1.6, 1.6),
                VolumeGrid(64, 64, 48, (1.0, 1.0, 1.0)), RampFilter.named("ramlak"))


def odd_case():
    """Odd, non-square sizes, off-centre volume, detector offsets and tilts."""
    scan = CircularScan(37, 36, 300.0, 650.0, 53, 41, 1.1, 0.9, start_angle_rad=0.2,
                        rotation_direction=-1, source_offset_mm=(0.7, -0.3, 0.4),
                        offset_unv_mm=(2.1, 0.0, -1.3), tilt_rad=(0.01, -0.015, 0.02))
    grid = VolumeGrid(29, 23, 19, (0.9, 1.1, 1.3), (1.5, -2.0, 0.75))
    return Case("odd-tilted", scan, grid, RampFilter.named("hann", cutoff=0.4), n_ellipsoids=5,
                seed=7, center_range=8.0, axis_min=2.0, axis_max=8.0)


def phantom(O, case: Case) -> np.ndarray:
    vol = O.volume_struct(case.grid.shape, case.grid.voxel_mm, case.grid.center_mm)
    ell = O.random_ellipsoids(case.seed, case.n_ellipsoids, case.center_range, case.axis_min,
                              case.axis_max)
    return O.voxelize(vol, ell)


def aligned_tilted():
    """odd_case's geometry with a detector the reference accepts (its row
    pitch and view size meet the texture alignment,
    src/Reconstruction/Analytic/Circular/Flat/FDK/YkFdkPipeline.hpp:283-301)."""
    scan = CircularScan(37, 36, 300.0, 650.0, 64, 40, 1.1, 0.9, start_angle_rad=0.2,
                        rotation_direction=-1, source_offset_mm=(0.7, -0.3, 0.4),
                        offset_unv_mm=(2.1, 0.0, -1.3), tilt_rad=(0.01, -0.015, 0.02))
    grid = VolumeGrid(29, 23, 19, (0.9, 1.1, 1.3), (1.5, -2.0, 0.75))
    return Case("tilted-aligned", scan, grid, RampFilter.named("hann", cutoff=0.4),
                n_ellipsoids=5, seed=7, center_range=8.0, axis_min=2.0, axis_max=8.0)


def smooth_projections(scan) -> np.ndarray:
    """Constant 1 plus a slow cosine: no texture weight quantisation effect
    at the 1e-6 level."""
    v = np.arange(scan.rows)[:, None] / scan.rows
    u = np.arange(scan.channels)[None, :] / scan.channels
    img = 1.0 + 0.05 * np.cos(np.pi * u) * np.cos(np.pi * v)
    return np.ascontiguousarray(np.broadcast_to(img, (scan.total_views, scan.rows, scan.channels)),
                                dtype=np.float32)


def oracle_volume(O, grid: VolumeGrid):
    return O.volume_struct(grid.shape, grid.voxel_mm, grid.center_mm)


def oracle_filter(O, f: RampFilter):
    return O.filter_struct(f.type, f.cutoff, f.gain, f.butterworth_order, f.kaiser_beta,
                           f.tukey_alpha)


def projections(O, case: Case, views=None, ph=None) -> np.ndarray:
    views = case.scan.views() if views is None else views
    ph = phantom(O, case) if ph is None else ph
    p = O.joseph_fp(views, case.scan.channels, case.scan.rows, oracle_volume(O, case.grid),
                    ph).astype(np.float32)
    if case.noise_i0:
        p = O.poisson_noise(p, case.noise_i0, case.seed + 100)
    return p


def rel_rmse(a, ref) -> float:
    a = np.asarray(a, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.sqrt(np.mean((a - ref) ** 2)) / max(np.sqrt(np.mean(ref ** 2)), 1e-300))


def cosine(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(a @ b / np.sqrt(max((a @ a) * (b @ b), 1e-300)))
