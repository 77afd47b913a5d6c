// Siddon projector pair (FP_Siddon, BP_Siddon_RayDriven): exact
// intersection lengths of the ray from the source to each detector pixel
// centre with the voxels it crosses.
//
// Same model as src/FlatFpBp/FP/kernels/YkFPSiddonKernel.cu:19-129 and
// src/FlatFpBp/BP/kernels/YkBPSiddonKernel.cu:31-127: the ray
// S + t (D - S), t in [0, 1], clipped to the volume's outer faces, entered at
// the voxel nearest its entry point, then walked voxel by voxel
// (Amanatides-Woo) with segment length (t_next - t) |D - S|.  Both kernels
// run the one walk below, so the backprojector is the exact transpose of the
// projector.
//
// Organised for the GPU: one thread per ray, 32 channels of a detector row
// per warp (neighbouring rays walk neighbouring voxels, so the gathers and
// the reductions hit the same L1/L2 lines).  The ray is set up in FP64 and
// walked in FP32 in mm from its entry point, each face crossing evaluated
// from its index (a + j d) instead of accumulated along the ray as the
// reference does over the whole source-detector parameter, so the split of
// the length between voxels does not drift over long rays.  The choice of
// axis is branch-free and the walk runs in batches of kBatch segments whose
// gathers are issued together.  The walk is bounded by nx + ny + nz + 3
// steps.  The backprojector adds each segment to
// its voxel with a global reduction (red.global.add.f32): the sum is exact
// up to FP32 rounding, in an order that varies from run to run, as the
// reference's atomicAdd.
#include "ykb_internal.hpp"

namespace ykb {
namespace {

struct SiddonRay {
    float smax;              // length of the ray inside the volume (mm)
    float len;               // |D - S| (mm)
    float aX, aY, aZ;        // distance from the entry to the next face on each axis
    float dX, dY, dZ;        // distance between consecutive faces on each axis
    float mX, mY, mZ;        // interior faces ahead on each axis (crossings allowed)
    int ix, iy, iz;          // entry voxel
    int sx, sy, sz;          // step directions
};

// slab clip of one axis; false when the ray misses
__device__ __forceinline__ bool clip_axis(double s, double r, double lo, double hi, double& tmin,
    double& tmax)
{
    if (fabs(r) > 1e-8) {
        double ta = (lo - s) / r, tb = (hi - s) / r;
        if (ta > tb) { const double t = ta; ta = tb; tb = t; }
        tmin = fmax(tmin, ta);
        tmax = fmin(tmax, tb);
        return true;
    }
    return s >= lo && s <= hi;
}

// entry voxel (nearest centre to the entry point), step direction, and the
// walk's distances along this axis, measured in mm from the entry point:
// the first face crossed at a, the following ones every d
__device__ __forceinline__ void axis_setup(double s, double r, double tmin, double len, double o,
    double v, int n, int& i, int& step, float& a, float& d, float& m)
{
    const double e = s + tmin * r;
    i = max(0, min(n - 1, static_cast<int>(floor((e - o) / v + 0.5))));
    step = r >= 0.0 ? 1 : -1;
    // faces between the entry voxel and the volume's far side: crossing
    // more would leave the volume, so the walk's indices stay in range
    m = static_cast<float>(step > 0 ? n - 1 - i : i);
    if (fabs(r) > 1e-8) {
        // face k lies at o + (k - 1/2) v
        const double k = step > 0 ? i + 1.0 : static_cast<double>(i);
        a = static_cast<float>(fmax(((o + (k - 0.5) * v - s) / r - tmin) * len, 0.0));
        d = static_cast<float>(v / fabs(r) * len);
    } else {
        a = 3e38f;  // never crossed
        d = 0.f;
        m = 0.f;
    }
    if (m == 0.f) a = 3e38f;
}

__device__ __forceinline__ bool siddon_setup(const ykb_cone_view& v, int iu, int iv,
    const VolumeGrid& g, SiddonRay& R)
{
    const double Sx = v.src.x, Sy = v.src.y, Sz = v.src.z;
    const double Dx = v.detS.x + iu * static_cast<double>(v.detU.x) + iv * static_cast<double>(v.detV.x);
    const double Dy = v.detS.y + iu * static_cast<double>(v.detU.y) + iv * static_cast<double>(v.detV.y);
    const double Dz = v.detS.z + iu * static_cast<double>(v.detU.z) + iv * static_cast<double>(v.detV.z);
    const double rx = Dx - Sx, ry = Dy - Sy, rz = Dz - Sz;
    const double len = sqrt(rx * rx + ry * ry + rz * rz);
    double tmin = 0.0, tmax = 1.0;
    if (!clip_axis(Sx, rx, g.ox - 0.5 * g.vx, g.ox + (g.nx - 0.5) * g.vx, tmin, tmax) ||
        !clip_axis(Sy, ry, g.oy - 0.5 * g.vy, g.oy + (g.ny - 0.5) * g.vy, tmin, tmax) ||
        !clip_axis(Sz, rz, g.oz - 0.5 * g.vz, g.oz + (g.nz - 0.5) * g.vz, tmin, tmax))
        return false;
    if (!(tmin < tmax)) return false;
    R.len = static_cast<float>(len);
    R.smax = static_cast<float>((tmax - tmin) * len);
    axis_setup(Sx, rx, tmin, len, g.ox, g.vx, g.nx, R.ix, R.sx, R.aX, R.dX, R.mX);
    axis_setup(Sy, ry, tmin, len, g.oy, g.vy, g.ny, R.iy, R.sy, R.aY, R.dY, R.mY);
    axis_setup(Sz, rz, tmin, len, g.oz, g.vz, g.nz, R.iz, R.sz, R.aZ, R.dZ, R.mZ);
    return true;
}

// Walks the ray in batches of kBatch segments: the walk of a batch is pure
// arithmetic, then f(index[], length[]) consumes it, so a thread has several
// independent gathers (or reductions) in flight.  Each axis crosses at most
// its interior faces ahead (mX, mY, mZ), after which its next face is at
// infinity: the voxel index never leaves the volume, and the walk ends when
// the distance reaches smax.  Segments past the exit have length 0 and the
// entry voxel's index.  I is the voxel index type (int below 2^31 voxels).
constexpr int kBatch = 4;

template <typename I, typename F>
__device__ __forceinline__ void siddon_walk(const SiddonRay& R, const VolumeGrid& g, F&& f)
{
    const I entry = (static_cast<I>(R.iz) * g.ny + R.iy) * g.nx + R.ix;
    const I stepX = R.sx, stepY = static_cast<I>(R.sy) * g.nx,
            stepZ = static_cast<I>(R.sz) * g.nx * g.ny;
    I idx = entry;
    float s = 0.f, sX = R.aX, sY = R.aY, sZ = R.aZ;
    float jx = 0.f, jy = 0.f, jz = 0.f;  // faces crossed so far (exact small integers)
    const int max_steps = g.nx + g.ny + g.nz + 3;
    for (int it = 0; it < max_steps && s < R.smax; it += kBatch) {
        I id[kBatch];
        float ds[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const bool inside = s < R.smax;
            // never behind s: an entry point on a face can round to the
            // voxel before it, whose far face then lies at s
            const float sn = fmaxf(s, fminf(fminf(sX, sY), fminf(sZ, R.smax)));
            ds[u] = inside ? sn - s : 0.f;
            id[u] = inside ? idx : entry;
            s = inside ? sn : R.smax;
            const bool xm = sX <= sY && sX <= sZ;
            const bool ym = !xm && sY <= sZ;
            idx += xm ? stepX : (ym ? stepY : stepZ);
            if (xm) {
                jx += 1.f;
                sX = jx < R.mX ? fmaf(jx, R.dX, R.aX) : 3e38f;
            } else if (ym) {
                jy += 1.f;
                sY = jy < R.mY ? fmaf(jy, R.dY, R.aY) : 3e38f;
            } else {
                jz += 1.f;
                sZ = jz < R.mZ ? fmaf(jz, R.dZ, R.aZ) : 3e38f;
            }
        }
        f(id, ds);
    }
}

template <typename I>
__global__ void __launch_bounds__(128) siddon_fp_kernel(const float* __restrict__ vol,
    const ykb_cone_view* __restrict__ views, int view0, int nu, int nv, VolumeGrid g,
    float* __restrict__ proj, int accumulate)
{
    const int iu = blockIdx.x * 32 + threadIdx.x;
    const int iv = blockIdx.y * 4 + threadIdx.y;
    const int k = view0 + blockIdx.z;
    if (iu >= nu || iv >= nv) return;
    SiddonRay R;
    float acc = 0.f;
    if (siddon_setup(views[k], iu, iv, g, R)) {
        siddon_walk<I>(R, g, [&](const I* id, const float* ds) {
            float x[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) x[u] = __ldg(vol + id[u]);
#pragma unroll
            for (int u = 0; u < kBatch; ++u) acc = fmaf(x[u], ds[u], acc);
        });
    }
    float* dst = proj + (static_cast<long>(k) * nv + iv) * nu + iu;
    *dst = accumulate ? *dst + acc : acc;
}

template <typename I>
__global__ void __launch_bounds__(128) siddon_bp_kernel(const float* __restrict__ proj,
    const ykb_cone_view* __restrict__ views, int view0, int nu, int nv, VolumeGrid g,
    float* __restrict__ vol)
{
    const int iu = blockIdx.x * 32 + threadIdx.x;
    const int iv = blockIdx.y * 4 + threadIdx.y;
    const int k = view0 + blockIdx.z;
    if (iu >= nu || iv >= nv) return;
    SiddonRay R;
    if (!siddon_setup(views[k], iu, iv, g, R)) return;
    const float p = proj[(static_cast<long>(k) * nv + iv) * nu + iu];
    if (p == 0.f) return;
    siddon_walk<I>(R, g, [&](const I* id, const float* ds) {
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (ds[u] != 0.f) atomicAdd(vol + id[u], p * ds[u]);
    });
}

bool small_volume(const VolumeGrid& g)
{
    return static_cast<long>(g.nx) * g.ny * g.nz < (1L << 31);
}

} // namespace

cudaError_t launch_siddon_fp(const float* vol, const ykb_cone_view* views, int n_views, int nu,
    int nv, const VolumeGrid& g, float* proj, int accumulate, cudaStream_t s)
{
    for (int done = 0; done < n_views; done += 65535) {
        const int count = min(n_views - done, 65535);
        const dim3 grid((nu + 31) / 32, (nv + 3) / 4, count);
        if (small_volume(g))
            siddon_fp_kernel<int><<<grid, dim3(32, 4), 0, s>>>(vol, views, done, nu, nv, g, proj, accumulate);
        else
            siddon_fp_kernel<long><<<grid, dim3(32, 4), 0, s>>>(vol, views, done, nu, nv, g, proj, accumulate);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_siddon_bp(const float* proj, const ykb_cone_view* views, int n_views, int nu,
    int nv, const VolumeGrid& g, float* vol, int accumulate, cudaStream_t s)
{
    if (!accumulate) {
        const cudaError_t e = cudaMemsetAsync(vol,
            0, static_cast<size_t>(g.nx) * g.ny * g.nz * sizeof(float), s);
        if (e != cudaSuccess) return e;
    }
    for (int done = 0; done < n_views; done += 65535) {
        const int count = min(n_views - done, 65535);
        const dim3 grid((nu + 31) / 32, (nv + 3) / 4, count);
        if (small_volume(g))
            siddon_bp_kernel<int><<<grid, dim3(32, 4), 0, s>>>(proj, views, done, nu, nv, g, vol);
        else
            siddon_bp_kernel<long><<<grid, dim3(32, 4), 0, s>>>(proj, views, done, nu, nv, g, vol);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

} // namespace ykb
