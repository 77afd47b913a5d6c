// Weight of the pseudo-matched backprojection (BP_FDK_PseudoMatched,
// src/FlatFpBp/BP/kernels/YkBpFdkKernel.cu:425-446): for a voxel P at
// detector coordinates (u, v) of a view with source S,
//     w = k L^3 / |P - S|^2,  L^2 = |detS + u detU + v detV - S|^2,
// k = voxel volume / (du dv |SDD_plane|).  This is the ray density of a
// line-integral projector at P (rays per unit area through a pixel of solid
// angle du dv SDD_plane / L^3, seen at distance |P - S|) times the voxel
// volume, the transpose of the projector up to its interpolation kernel.
#pragma once

#include "ykb_internal.hpp"

namespace ykb {

// |P(i) - S|^2 = q0 + i (q1 + i q2) along a z-column P(i) = (X, Y, Z0 + i vz)
struct PseudoColumn {
    float q0, q1, q2;
};

__device__ __forceinline__ PseudoColumn pseudo_column(const PseudoViewCoef& p, double X,
    double Y, double Z0, double vz)
{
    const double dx = X - p.src[0], dy = Y - p.src[1], dz = Z0 - p.src[2];
    PseudoColumn c;
    c.q0 = static_cast<float>(dx * dx + dy * dy + dz * dz);
    c.q1 = static_cast<float>(2.0 * dz * vz);
    c.q2 = static_cast<float>(vz * vz);
    return c;
}

__device__ __forceinline__ float pseudo_weight(const PseudoViewCoef& p, const PseudoColumn& c,
    float fi, float u, float v)
{
    const float lsq = fmaf(fi, fmaf(fi, c.q2, c.q1), c.q0);
    const float L2 = fmaf(v, fmaf(v, p.l2[5], fmaf(u, p.l2[4], p.l2[2])),
                          fmaf(u, fmaf(u, p.l2[3], p.l2[1]), p.l2[0]));
    // the reference skips voxels with L^2 or |P - S|^2 below 1e-8
    if (!(L2 > 1e-8f) || !(lsq > 1e-8f)) return 0.f;
    return p.k * (L2 * __fsqrt_rn(L2)) * __frcp_rn(lsq);
}

} // namespace ykb
