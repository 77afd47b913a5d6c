"""Seeded synthetic FDK workloads of the benchmark and the full-size tests.

Each workload is a flat-panel circular scan (source-to-isocentre 500 mm,
source-to-detector 1000 mm), a cubic volume, and an ellipsoid phantom
projected by the Joseph forward projector, with optional Poisson noise:

  c2     512^3 of 0.25 mm, 720 views, 768^2 detector of 0.4 mm, 20 ellipsoids,
         noise at 1e5 photons, FP32 projections (the headline workload)
  large  1024^3 of 0.125 mm, 1440 views, 1536^2 of 0.2 mm, 40 ellipsoids and
         200 spheres (radius 0.5-2 mm, attenuation 2.0), noise-free, projections
         stored in BF16 (6.8 GB)
  small  256^3 of 0.5 mm, 360 views, 384^2 of 0.8 mm (inputs still larger than
         L2), for profiler captures
  det768 256^3 of 0.5 mm, 96 views, the 768^2 detector of c2: the filter's
         row length of the headline workload at a small view count, for
         profiler captures
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geometry import CircularScan, VolumeGrid

SID_MM, SDD_MM = 500.0, 1000.0


@dataclass(frozen=True)
class FdkWorkload:
    name: str
    n_vox: int
    n_views: int
    n_det: int
    vox_mm: float
    pix_mm: float
    n_ellipsoids: int
    n_spheres: int
    noise_i0: float | None
    projections: str  # "f32" or "bf16": how the projections are stored

    def scan(self) -> CircularScan:
        return CircularScan(self.n_views, self.n_views, SID_MM, SDD_MM, self.n_det, self.n_det,
                            self.pix_mm, self.pix_mm)

    def grid(self) -> VolumeGrid:
        return VolumeGrid.cube(self.n_vox, self.vox_mm)

    @property
    def updates(self) -> int:
        """Voxel x view updates of one backprojection of all views."""
        return self.n_vox ** 3 * self.n_views

    @property
    def label(self) -> str:
        return (f"fdk-{self.n_vox}^3-{self.n_views}v-{self.n_det}^2" +
                ("-bf16" if self.projections == "bf16" else ""))

    def describe(self) -> dict:
        """The workload's parameters, as the benchmark reports them."""
        return {"workload": self.label, "volume": [self.n_vox] * 3, "voxel_mm": self.vox_mm,
                "views": self.n_views, "detector": [self.n_det, self.n_det],
                "pixel_mm": self.pix_mm, "sid_sdd_mm": [SID_MM, SDD_MM],
                "ellipsoids": self.n_ellipsoids, "spheres": self.n_spheres,
                "noise_i0": self.noise_i0, "projections": self.projections}


WORKLOADS = {
    "c2": FdkWorkload("c2", 512, 720, 768, 0.25, 0.4, 20, 0, 1e5, "f32"),
    "large": FdkWorkload("large", 1024, 1440, 1536, 0.125, 0.2, 40, 200, None, "bf16"),
    "small": FdkWorkload("small", 256, 360, 384, 0.5, 0.8, 20, 0, 1e5, "f32"),
    "det768": FdkWorkload("det768", 256, 96, 768, 0.5, 0.4, 20, 0, 1e5, "f32"),
}


def phantom_objects(w: FdkWorkload, seed: int) -> np.ndarray:
    from . import phantom as PH
    ell = PH.random_ellipsoids(seed, w.n_ellipsoids)
    if w.n_spheres:
        ell = np.concatenate([ell, PH.random_spheres(seed, w.n_spheres)])
    return ell


def make_projections(w: FdkWorkload, seed: int, device: int = 0, forward=None, views=None,
                     chunk_views: int | None = None):
    """(views, projections) of workload w on cuda:device: the seeded phantom,
    forward projected in view chunks, noise added in FP64 and the result
    stored as w.projections.  `forward(views_chunk, phantom)` returns a
    float32 CUDA tensor [n][n_det][n_det]; the default is this package's
    Joseph projector, in chunks of at most 4 GiB of its ray records.  `views`
    (default: the scan's, from this package's builder) and `chunk_views`
    serve other projectors."""
    import torch
    from . import phantom as PH
    scan, grid = w.scan(), w.grid()
    if views is None:
        views = scan.views()
    phantom = PH.voxelize(grid, phantom_objects(w, seed), device=f"cuda:{device}")
    if forward is None:
        from .projectors import JosephPlan

        def forward(vchunk, vol):
            jp = JosephPlan(vchunk, w.n_det, w.n_det, grid, device=device)
            try:
                return jp.forward(vol)
            finally:
                jp.close()
    dtype = torch.bfloat16 if w.projections == "bf16" else torch.float32
    proj = torch.empty((w.n_views, w.n_det, w.n_det), dtype=dtype, device=f"cuda:{device}")
    # the projector's plan holds a 20-byte ray record per detector pixel of
    # its views: chunks of at most 4 GiB of records
    step = chunk_views or max(1, min(w.n_views, (4 << 30) // (20 * w.n_det * w.n_det)))
    for v0 in range(0, w.n_views, step):
        part = forward(views[v0:v0 + step], phantom)
        if w.noise_i0 is not None:
            PH.poisson_noise_(part, w.noise_i0, seed=7 + seed + v0)
        proj[v0:v0 + step] = part
        del part
    del phantom
    torch.cuda.synchronize(device)
    torch.cuda.empty_cache()
    return views, proj


def slab(w: FdkWorkload, z0: int, nz: int):
    """The VolumeGrid of slices [z0, z0 + nz) of w's volume."""
    g = w.grid()
    zc = g.center_mm[2] + (z0 + 0.5 * (nz - 1) - 0.5 * (g.nz - 1)) * g.voxel_mm[2]
    return VolumeGrid(g.nx, g.ny, nz, g.voxel_mm, (g.center_mm[0], g.center_mm[1], zc))
