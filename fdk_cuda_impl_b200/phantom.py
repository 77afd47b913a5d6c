"""Seeded synthetic inputs on the GPU: ellipsoid phantoms and Poisson noise.

Ellipsoids: centres U[-r, r], semi-axes U[a0, a1], rotation R = Rz(phi)
Ry(theta) Rz(psi) with angles U[0, 2pi), additive attenuation U[v0, v1];
voxelised by sampling voxel centres.  Noise: p' = -ln(max(Poisson(I0
exp(-p)), 1) / I0).
"""
from __future__ import annotations

import numpy as np
import torch

from .geometry import VolumeGrid


def random_ellipsoids(seed: int, count: int, center_range=25.0, axis_min=3.0, axis_max=25.0,
                      value_min=-0.2, value_max=1.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    e = np.empty((count, 10))
    e[:, 0:3] = rng.uniform(-center_range, center_range, (count, 3))
    e[:, 3:6] = rng.uniform(axis_min, axis_max, (count, 3))
    e[:, 6:9] = rng.uniform(0.0, 2 * np.pi, (count, 3))
    e[:, 9] = rng.uniform(value_min, value_max, count)
    return e


def random_spheres(seed: int, count: int, center_range=60.0, radius_min=0.5, radius_max=2.0,
                   value=2.0) -> np.ndarray:
    rng = np.random.default_rng(seed + 7919)
    e = np.zeros((count, 10))
    e[:, 0:3] = rng.uniform(-center_range, center_range, (count, 3))
    r = rng.uniform(radius_min, radius_max, count)
    e[:, 3] = e[:, 4] = e[:, 5] = r
    e[:, 9] = value
    return e


def _rotation(phi, theta, psi):
    c1, s1, c2, s2, c3, s3 = np.cos(phi), np.sin(phi), np.cos(theta), np.sin(theta), np.cos(psi), np.sin(psi)
    return np.array([[c1 * c2 * c3 - s1 * s3, -c1 * c2 * s3 - s1 * c3, c1 * s2],
                     [s1 * c2 * c3 + c1 * s3, -s1 * c2 * s3 + c1 * c3, s1 * s2],
                     [-s2 * c3, s2 * s3, c2]])


def voxelize(grid: VolumeGrid, ellipsoids: np.ndarray, device="cuda", slab: int = 32) -> torch.Tensor:
    """Centre-sampled sum of ellipsoid indicator functions, float32 [nz][ny][nx]."""
    out = torch.zeros(grid.shape, dtype=torch.float32, device=device)
    vx, vy, vz = grid.voxel_mm
    cx, cy, cz = grid.center_mm
    xs = cx + (torch.arange(grid.nx, device=device, dtype=torch.float64) - 0.5 * (grid.nx - 1)) * vx
    ys = cy + (torch.arange(grid.ny, device=device, dtype=torch.float64) - 0.5 * (grid.ny - 1)) * vy
    for z0 in range(0, grid.nz, slab):
        z1 = min(grid.nz, z0 + slab)
        zs = cz + (torch.arange(z0, z1, device=device, dtype=torch.float64) - 0.5 * (grid.nz - 1)) * vz
        acc = torch.zeros((z1 - z0, grid.ny, grid.nx), dtype=torch.float64, device=device)
        for e in ellipsoids:
            # only the voxels within the largest semi-axis of the centre can
            # be inside: q >= |d|^2 / a_max^2 > 1 beyond it
            box = []
            for c, axis_mm, n, origin in ((e[2], vz, z1 - z0, zs[0].item()), (e[1], vy, grid.ny, ys[0].item()),
                                          (e[0], vx, grid.nx, xs[0].item())):
                r = max(e[3], e[4], e[5])
                lo = max(0, int(np.floor((c - r - origin) / axis_mm)) - 1)
                hi = min(n, int(np.ceil((c + r - origin) / axis_mm)) + 2)
                box.append((lo, hi))
            (za, zb), (ya, yb), (xa, xb) = box
            if za >= zb or ya >= yb or xa >= xb:
                continue
            Z, Y, X = torch.meshgrid(zs[za:zb], ys[ya:yb], xs[xa:xb], indexing="ij")
            R = torch.as_tensor(_rotation(e[6], e[7], e[8]), device=device)
            dx, dy, dz = X - e[0], Y - e[1], Z - e[2]
            lx = R[0, 0] * dx + R[1, 0] * dy + R[2, 0] * dz
            ly = R[0, 1] * dx + R[1, 1] * dy + R[2, 1] * dz
            lz = R[0, 2] * dx + R[1, 2] * dy + R[2, 2] * dz
            q = (lx / e[3]) ** 2 + (ly / e[4]) ** 2 + (lz / e[5]) ** 2
            acc[za:zb, ya:yb, xa:xb] += torch.where(q <= 1.0, e[9], 0.0)
        out[z0:z1] = acc.float()
    return out


def poisson_noise_(proj: torch.Tensor, i0: float, seed: int) -> torch.Tensor:
    """In place: p <- -ln(max(Poisson(I0 exp(-p)), 1) / I0)."""
    g = torch.Generator(device=proj.device).manual_seed(seed)
    for k in range(proj.shape[0]):
        lam = i0 * torch.exp(-proj[k].double())
        counts = torch.poisson(lam, generator=g).clamp_min(1.0)
        proj[k] = (-torch.log(counts / i0)).float()
    return proj
