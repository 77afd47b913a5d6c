// Joseph forward projector and its exact matched backprojector for sm_100a.
//
// Discretisation (src/FlatFpBp/FP/kernels/YkFPKernels.cu:10-202): a ray from
// the source through pixel centre (u,v) is sampled once per voxel centre of
// the view's main axis; each sample is the bilinear interpolation of that
// slice on the two minor axes with zero outside the volume; the ray sum is
// scaled by the chord length per step sqrt(v0^2 + (a1 v1)^2 + (a2 v2)^2).
// The backprojector applies the transpose of exactly these weights,
// gathering per voxel over the rays that touch it (no atomics), where the
// reference scatters with four atomicAdd per sample
// (src/FlatFpBp/BP/kernels/YkBPJosephKernel.cu:12-113).
#include "ykb_internal.hpp"

namespace ykb {
namespace {

// Ray parameters shared bit-for-bit by the forward projector and the ray
// table of the backprojector: slopes a1,a2 and offsets e1,e2 such that the
// minor-axis voxel-index coordinates at main-axis slice s are
//   f1 = fmaf(a1, c0, e1), f2 = fmaf(a2, c0, e2), c0 = s - (n0-1)/2,
// plus the chord length per step.  Evaluated in FP64, rounded once.
struct RayParams { float a1, e1, a2, e2, len; bool ok; };

__device__ __forceinline__ double comp(const double* p, int axis, int which)
{
    // (main, minor1, minor2) permutation of AxisX/AxisY/AxisZ
    // (src/common/cuda/operators/YkOperatorKernelTypes.cuh:212-275)
    const int k = axis == 0 ? which : axis == 1 ? (which == 0 ? 1 : which == 1 ? 0 : 2)
                                                : (which == 0 ? 2 : which == 1 ? 0 : 1);
    return p[k];
}

__device__ __forceinline__ RayParams ray_params(const JosephView& j, int iu, int iv)
{
    double det[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) det[c] = j.detS[c] + iu * j.detU[c] + iv * j.detV[c];
    RayParams r{};
    const double s0 = comp(j.src, j.axis, 0), s1 = comp(j.src, j.axis, 1), s2 = comp(j.src, j.axis, 2);
    const double dc0 = s0 - comp(det, j.axis, 0);
    if (fabs(dc0) < 1e-12) { r.ok = false; return r; }
    const double a1 = (s1 - comp(det, j.axis, 1)) / dc0;
    const double a2 = (s2 - comp(det, j.axis, 2)) / dc0;
    const double b1 = s1 - a1 * s0, b2 = s2 - a2 * s0;
    const double a1v1 = a1 * j.v1, a2v2 = a2 * j.v2;
    r.a1 = static_cast<float>(a1);
    r.a2 = static_cast<float>(a2);
    r.e1 = static_cast<float>(b1 + 0.5 * (j.n1 - 1));
    r.e2 = static_cast<float>(b2 + 0.5 * (j.n2 - 1));
    r.len = static_cast<float>(sqrt(j.v0 * j.v0 + a1v1 * a1v1 + a2v2 * a2v2));
    r.ok = true;
    return r;
}

// Slices s where the sample can touch the volume: -1 < f < n on both minor
// axes (conservatively widened by one slice each side).
__device__ __forceinline__ void slice_range(float a, float e, int n, int n0, int& lo, int& hi)
{
    const float h = 0.5f * (n0 - 1);
    if (fabsf(a) < 1e-12f) {
        if (!(e > -1.f && e < static_cast<float>(n))) { lo = 1; hi = 0; }
        return;
    }
    float t0 = (-1.f - e) / a + h, t1 = (static_cast<float>(n) - e) / a + h;
    if (t0 > t1) { const float t = t0; t0 = t1; t1 = t; }
    // clamp before the integer conversion (NaN compares false and stays put)
    t0 = fminf(fmaxf(t0, -1e7f), 1e7f);
    t1 = fminf(fmaxf(t1, -1e7f), 1e7f);
    lo = max(lo, static_cast<int>(floorf(t0)) - 1);
    hi = min(hi, static_cast<int>(ceilf(t1)) + 1);
}

// Slices where f = a (s - (n0 - 1)/2) + e lies in [-3/2, n + 1/2], in FP64
// from the float a and e the kernels evaluate: they hold every sample with
// a non-zero weight (-1 < f < n), and the float f of each of them is within
// an ulp of that interval, so its floor is in [-2, n] and both taps are
// inside a two-voxel border.
__device__ __forceinline__ void slice_range_border(float a, float e, int n, int n0, int& lo,
    int& hi)
{
    const double L = -1.5, U = static_cast<double>(n) + 0.5, h = 0.5 * (n0 - 1);
    const double ad = a, ed = e;
    if (fabs(ad) < 1e-300) {
        if (!(ed >= L && ed <= U)) { lo = 1; hi = 0; }
        return;
    }
    double t0 = (L - ed) / ad + h, t1 = (U - ed) / ad + h;
    if (t0 > t1) { const double t = t0; t0 = t1; t1 = t; }
    t0 = fmin(fmax(t0, -1e9), 1e9);
    t1 = fmin(fmax(t1, -1e9), 1e9);
    lo = max(lo, static_cast<int>(ceil(t0)));
    hi = min(hi, static_cast<int>(floor(t1)));
}

// One thread per ray; a block covers 32 channels x 4 rows of one view, a
// warp one detector row.  The warp walks the union of its rays' slice ranges
// together, each lane sampling only inside its own: at every step the 32
// gathers fall on one slice plane, on a run of about 32 magnified voxels of
// two rows, instead of on up to a few planes when lanes whose rays enter
// the volume at different slices would run ahead of one another.  Each
// lane's samples and their order are unchanged.
__global__ void __launch_bounds__(128) joseph_fp_kernel(const float* __restrict__ slab,
    const JosephView* __restrict__ views, int view0, int nu, int nv, float* __restrict__ proj,
    int accumulate)
{
    const int iu = blockIdx.x * 32 + threadIdx.x;
    const int iv = blockIdx.y * 4 + threadIdx.y;
    const int k = view0 + blockIdx.z;
    const bool pixel = iu < nu && iv < nv;
    const JosephView& j = views[k];
    const RayParams r = ray_params(j, min(iu, nu - 1), min(iv, nv - 1));
    int lo = 0, hi = j.n0 - 1;
    if (pixel && r.ok) {
        slice_range(r.a1, r.e1, j.n1, j.n0, lo, hi);
        slice_range(r.a2, r.e2, j.n2, j.n0, lo, hi);
    } else {
        lo = 1; hi = 0;
    }
    // the warp's slice span (every lane reaches here: no early return above)
    const int wlo = __reduce_min_sync(0xffffffffu, lo <= hi ? lo : 0x7fffffff);
    const int whi = __reduce_max_sync(0xffffffffu, lo <= hi ? hi : -1);
    // FP64 ray sum: keeps the adjoint identity at the 1e-7 level
    double acc = 0.0;
    {
        const long plane = static_cast<long>(j.n1) * j.n2;
        const float half = 0.5f * (j.n0 - 1);
        // unrolled: the four gathers of several samples are in flight at once
#pragma unroll 4
        for (int s = wlo; s <= whi; ++s) {
            if (s < lo || s > hi) continue;
            const float c0 = static_cast<float>(s) - half;
            const float f1 = fmaf(r.a1, c0, r.e1);
            const float f2 = fmaf(r.a2, c0, r.e2);
            const float fl1 = floorf(f1), fl2 = floorf(f2);
            const int i1 = static_cast<int>(fl1), i2 = static_cast<int>(fl2);
            const float w1 = f1 - fl1, w2 = f2 - fl2;
            const float* sl = slab + s * plane;
            const bool c1a = static_cast<unsigned>(i1) < static_cast<unsigned>(j.n1);
            const bool c1b = static_cast<unsigned>(i1 + 1) < static_cast<unsigned>(j.n1);
            const bool c2a = static_cast<unsigned>(i2) < static_cast<unsigned>(j.n2);
            const bool c2b = static_cast<unsigned>(i2 + 1) < static_cast<unsigned>(j.n2);
            const long ra = static_cast<long>(i2) * j.n1, rb = ra + j.n1;
            const float p00 = (c1a && c2a) ? __ldg(sl + ra + i1) : 0.f;
            const float p10 = (c1b && c2a) ? __ldg(sl + ra + i1 + 1) : 0.f;
            const float p01 = (c1a && c2b) ? __ldg(sl + rb + i1) : 0.f;
            const float p11 = (c1b && c2b) ? __ldg(sl + rb + i1 + 1) : 0.f;
            acc += static_cast<double>((1.f - w2) * ((1.f - w1) * p00 + w1 * p10) +
                w2 * ((1.f - w1) * p01 + w1 * p11));
        }
        acc *= r.len;
    }
    if (!pixel) return;
    float* dst = proj + (static_cast<long>(k) * nv + iv) * nu + iu;
    *dst = accumulate ? static_cast<float>(*dst + acc) : static_cast<float>(acc);
}

// Packed FP32 pairs (sm_100 f32x2 arithmetic): both minor axes at once.
typedef unsigned long long f2;
__device__ __forceinline__ f2 f2pack(float lo, float hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2unpack(f2 v, float& lo, float& hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 f2fma(f2 a, f2 b, f2 c)
{
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2 f2add(f2 a, f2 b)
{
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2sub(f2 a, f2 b)
{
    f2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// 1.5 * 2^23: for |x| < 2^22, x + kMagic holds round(x) in its low mantissa
// bits; (f - 1/2) + kMagic thus holds floor(f), except at integer f where
// it may hold f - 1 -- with fraction 1, the same bilinear weights.
constexpr float kMagic = 12582912.0f;
constexpr uint32_t kMagicBits = 0x4B400000u;

// The forward projector for main axis x or y, over the zero-bordered slabs
// (kSlabPad voxels each side of both minor axes).  The same samples and
// weights as joseph_fp_kernel, without per-tap bounds checks: each lane's
// slices are those where both minor coordinates lie in [-3/2, n + 1/2]
// (slice_range_border), so its four taps are inside the slab's border.
// Floor and fraction come from the
// rounding constant (both axes in one packed add each), the sample is the
// bilinear lerp of the four taps, added to the FP64 ray sum.  Lanes walk
// the warp's slice span together (see joseph_fp_kernel); a slice outside a
// lane's own range yields zero.
__global__ void __launch_bounds__(128) joseph_fp_padded_kernel(const float* __restrict__ slab,
    const JosephView* __restrict__ views, int view0, int nu, int nv, float* __restrict__ proj,
    int accumulate)
{
    const int iu = blockIdx.x * 32 + threadIdx.x;
    const int iv = blockIdx.y * 4 + threadIdx.y;
    const int k = view0 + blockIdx.z;
    const bool pixel = iu < nu && iv < nv;
    const JosephView& j = views[k];
    const RayParams r = ray_params(j, min(iu, nu - 1), min(iv, nv - 1));
    int lo = 0, hi = j.n0 - 1;
    if (pixel && r.ok) {
        slice_range_border(r.a1, r.e1, j.n1, j.n0, lo, hi);
        slice_range_border(r.a2, r.e2, j.n2, j.n0, lo, hi);
    } else {
        lo = 1; hi = 0;
    }
    const int wlo = __reduce_min_sync(0xffffffffu, lo <= hi ? lo : 0x7fffffff);
    const int whi = __reduce_max_sync(0xffffffffu, lo <= hi ? hi : -1);
    const int p1 = j.n1 + 2 * kSlabPad;
    const long plane = static_cast<long>(p1) * (j.n2 + 2 * kSlabPad);
    // element (i2, i1) of a slice at word (i2 + pad) p1 + i1 + pad, from the
    // rounding words t1, t2 of floor(f1), floor(f2) (wrapping arithmetic);
    // never past the slice's last 2x2 taps
    const uint32_t koff = static_cast<uint32_t>(kSlabPad) * static_cast<uint32_t>(p1 + 1) -
        kMagicBits * static_cast<uint32_t>(p1 + 1);
    const uint32_t last = static_cast<uint32_t>(plane) - static_cast<uint32_t>(p1) - 2u;
    const f2 A = f2pack(r.a1, r.a2), E = f2pack(r.e1, r.e2);
    const f2 H = f2pack(0.5f, 0.5f), M = f2pack(kMagic, kMagic);
    float c0 = static_cast<float>(wlo) - 0.5f * (j.n0 - 1);  // exact: integers and halves
    // FP64 ray sum: keeps the adjoint identity at the 1e-7 level even where
    // <Ax, y> cancels to 1e-4 of its terms
    double acc = 0.0;
    // unrolled: the four gathers of several samples are in flight at once
#pragma unroll 4
    for (int sq = wlo; sq <= whi; ++sq, c0 += 1.f) {
        // a slice outside this lane's range reads the zero border corner
        const bool in = sq >= lo && sq <= hi;
        const f2 f = f2fma(A, f2pack(c0, c0), E);
        const f2 t = f2add(f2sub(f, H), M);
        float t1, t2, w1, w2;
        f2unpack(t, t1, t2);
        f2unpack(f2sub(f, f2sub(t, M)), w1, w2);
        const uint32_t off = in ? min(__float_as_uint(t2) * static_cast<uint32_t>(p1) +
            __float_as_uint(t1) + koff, last) : 0u;
        const float* p = slab + sq * plane + off;
        const float p00 = __ldg(p), p10 = __ldg(p + 1);
        const float p01 = __ldg(p + p1), p11 = __ldg(p + p1 + 1);
        const float a = fmaf(w1, p10 - p00, p00);
        const float b = fmaf(w1, p11 - p01, p01);
        acc += static_cast<double>(fmaf(w2, b - a, a));
    }
    acc *= r.len;
    if (!pixel) return;
    float* dst = proj + (static_cast<long>(k) * nv + iv) * nu + iu;
    *dst = accumulate ? static_cast<float>(*dst + acc) : static_cast<float>(acc);
}

__global__ void __launch_bounds__(128) joseph_ray_table_kernel(const JosephView* __restrict__ views,
    int nu, int nv, float4* __restrict__ rays, float* __restrict__ lens)
{
    const int iu = blockIdx.x * 32 + threadIdx.x;
    const int iv = blockIdx.y * 4 + threadIdx.y;
    const int k = blockIdx.z;
    if (iu >= nu || iv >= nv) return;
    const RayParams r = ray_params(views[k], iu, iv);
    const long idx = (static_cast<long>(k) * nv + iv) * nu + iu;
    rays[idx] = r.ok ? make_float4(r.a1, r.e1, r.a2, r.e2) : make_float4(0.f, -1e30f, 0.f, -1e30f);
    lens[idx] = r.ok ? r.len : 0.f;
}

// vol[z][y][x] -> slab[y][z][x] (main axis Y) and slab[x][z][y] (main axis X),
// each slice bordered by kSlabPad zero voxels on both minor axes (the
// borders are zeroed once, when the plan is built, and never written here)
__global__ void transpose_yzx_kernel(const float* __restrict__ in, int nx, int ny, int nz,
    float* __restrict__ out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    const long row = static_cast<long>(y) * (nz + 2 * kSlabPad) + z + kSlabPad;
    out[row * (nx + 2 * kSlabPad) + x + kSlabPad] = in[(static_cast<long>(z) * ny + y) * nx + x];
}

__global__ void transpose_xzy_kernel(const float* __restrict__ in, int nx, int ny, int nz,
    float* __restrict__ out)
{
    __shared__ float tile[32][33];
    const int z = blockIdx.z;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int y = y0 + r, x = x0 + threadIdx.x;
        tile[r][threadIdx.x] = (x < nx && y < ny) ? in[(static_cast<long>(z) * ny + y) * nx + x] : 0.f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int x = x0 + r, y = y0 + threadIdx.x;
        const long row = static_cast<long>(x) * (nz + 2 * kSlabPad) + z + kSlabPad;
        if (x < nx && y < ny) out[row * (ny + 2 * kSlabPad) + y + kSlabPad] = tile[threadIdx.x][r];
    }
}

// ---------------------------------------------------------------------------
// Matched backprojector, voxel-driven.  For voxel (s, j1, j2) in a view's
// main-axis frame the rays with a non-zero weight are those whose sample on
// slice s lies within one voxel of (j1, j2) on both minor axes; their pixels
// lie in the detector image of the square [j1-1,j1+1]x[j2-1,j2+1] on that
// slice, found from its four projected corners.  Each candidate's sample
// position is recomputed from the shared ray table with the forward
// projector's exact arithmetic, so the weights are those of joseph_fp_kernel.
// ---------------------------------------------------------------------------
struct ViewProj { float m[12]; };  // (u*w, v*w, w) = M (x', y', z', 1)

// Ray values weighted by their chord length: the backprojector gathers
// value * len * (bilinear weight) per ray, and this pass forms value * len
// once per ray instead of once per (voxel, ray) hit.
__global__ void joseph_weight_rays_kernel(const float* __restrict__ proj,
    const float* __restrict__ lens, long n, float* __restrict__ out)
{
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x)
        out[i] = proj[i] * lens[i];
}

// Weight with which a sample at minor coordinate f reaches voxel j:
// max(0, 1 - |f - j|).  The forward projector gives voxel floor(f) the weight
// 1 - w and voxel floor(f) + 1 the weight w, w = f - floor(f).  For
// floor(f) = j the expression is 1 - (f - j), the same operations.  For
// floor(f) = j - 1 it is 1 - (j - f): j - f = 1 - w is exact whenever
// f >= j / 2 (Sterbenz), i.e. for every j >= 2, and then 1 - (1 - w) = w
// exactly; at j = 0 (f in [-1, 0)) both compute f + 1.  Only j = 1 with
// f < 1/2 may differ, by one rounding of a weight below 1/2.
__device__ __forceinline__ float hat_weight(float f, float jf)
{
    return fmaxf(0.f, 1.f - fabsf(f - jf));
}

// Detector box of the slice rectangle [j1lo - 1, j1hi + 1] x [j2lo - 1,
// j2hi + 1] (voxel-index coordinates on the minor axes of slice c0), from its
// four projected corners, clipped to the detector; empty when u0 > u1 or
// v0 > v1.  The box of a sub-rectangle lies inside (the map is projective,
// the rectangle convex, and the 0.05-pixel margin covers the rounding).
__device__ __forceinline__ void footprint_box_range(const ViewProj& m, const JosephView& j,
    float c0, int j1lo, int j1hi, int j2lo, int j2hi, int nu, int nv, int& u0, int& u1, int& v0,
    int& v1)
{
    float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
#pragma unroll
    for (int corner = 0; corner < 4; ++corner) {
        const float q1 = static_cast<float>((corner & 1) ? j1hi + 1 : j1lo - 1) - 0.5f * (j.n1 - 1);
        const float q2 = static_cast<float>((corner & 2) ? j2hi + 1 : j2lo - 1) - 0.5f * (j.n2 - 1);
        float px, py, pz;
        if (j.axis == 0) { px = c0; py = q1; pz = q2; }
        else if (j.axis == 1) { px = q1; py = c0; pz = q2; }
        else { px = q1; py = q2; pz = c0; }
        const float w = fmaf(m.m[8], px, fmaf(m.m[9], py, fmaf(m.m[10], pz, m.m[11])));
        // the box only needs a few 1e-6 px: correctly rounded reciprocal
        const float rw = __frcp_rn(w);
        const float u = fmaf(m.m[0], px, fmaf(m.m[1], py, fmaf(m.m[2], pz, m.m[3]))) * rw;
        const float v = fmaf(m.m[4], px, fmaf(m.m[5], py, fmaf(m.m[6], pz, m.m[7]))) * rw;
        umin = fminf(umin, u); umax = fmaxf(umax, u);
        vmin = fminf(vmin, v); vmax = fmaxf(vmax, v);
    }
    constexpr float margin = 0.05f;
    u0 = max(0, static_cast<int>(ceilf(umin - margin)));
    u1 = min(nu - 1, static_cast<int>(floorf(umax + margin)));
    v0 = max(0, static_cast<int>(ceilf(vmin - margin)));
    v1 = min(nv - 1, static_cast<int>(floorf(vmax + margin)));
}

// the box of [j1 - 1, j1 + 1] x [j2lo - 1, j2hi + 1]
__device__ __forceinline__ void footprint_box(const ViewProj& m, const JosephView& j, float c0,
    int j1, int j2lo, int j2hi, int nu, int nv, int& u0, int& u1, int& v0, int& v1)
{
    footprint_box_range(m, j, c0, j1, j1, j2lo, j2hi, nu, nv, u0, u1, v0, v1);
}

// One thread gathers ZV voxels stacked along z.  When z is a minor axis of
// the view (main axis x or y, every view of a circular orbit) the stack lies
// in one slice with a common minor-1 index: each candidate ray of the stack's
// detector box is loaded once, its minor-1 weight computed once, and only the
// minor-2 weight is evaluated per voxel.  Views whose main axis is z take
// the voxels one at a time.
template <int ZV>
__global__ void __launch_bounds__(256) joseph_bp_kernel(const float* __restrict__ vl,
    const float4* __restrict__ rays, const ViewProj* __restrict__ vp,
    const JosephView* __restrict__ views, int n_views, int nu, int nv, int nx, int ny, int nz,
    float* __restrict__ vol, int accumulate)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * ZV;
    if (x >= nx || y >= ny) return;
    const int view_elems = nu * nv;
    double acc[ZV];  // FP64 over views; each view's few hits summed in FP32
#pragma unroll
    for (int q = 0; q < ZV; ++q) acc[q] = 0.0;
    for (int k = 0; k < n_views; ++k) {
        const JosephView& j = views[k];
        const ViewProj& m = vp[k];
        const float4* rk = rays + static_cast<long>(k) * view_elems;
        const float* vk = vl + static_cast<long>(k) * view_elems;
        if (j.axis != 2) {
            const int s = j.axis == 0 ? x : y, j1 = j.axis == 0 ? y : x;
            const float c0 = static_cast<float>(s) - 0.5f * (j.n0 - 1);
            int u0, u1, v0, v1;
            footprint_box(m, j, c0, j1, z0, z0 + ZV - 1, nu, nv, u0, u1, v0, v1);
            const float j1f = static_cast<float>(j1);
            float jq[ZV], accv[ZV];
#pragma unroll
            for (int q = 0; q < ZV; ++q) { jq[q] = static_cast<float>(z0 + q); accv[q] = 0.f; }
            for (int iv = v0; iv <= v1; ++iv) {
                const int row = iv * nu;
                for (int iu = u0; iu <= u1; ++iu) {
                    const float4 r = __ldg(rk + row + iu);
                    const float t = __ldg(vk + row + iu) * hat_weight(fmaf(r.x, c0, r.y), j1f);
                    const float f2 = fmaf(r.z, c0, r.w);
#pragma unroll
                    for (int q = 0; q < ZV; ++q) accv[q] = fmaf(t, hat_weight(f2, jq[q]), accv[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < ZV; ++q) acc[q] += static_cast<double>(accv[q]);
        } else {
            // main axis z: each voxel of the stack is its own slice
            const float j1f = static_cast<float>(x), j2f = static_cast<float>(y);
#pragma unroll
            for (int q = 0; q < ZV; ++q) {
                const float c0 = static_cast<float>(z0 + q) - 0.5f * (j.n0 - 1);
                int u0, u1, v0, v1;
                footprint_box(m, j, c0, x, y, y, nu, nv, u0, u1, v0, v1);
                float accv = 0.f;
                for (int iv = v0; iv <= v1; ++iv) {
                    const int row = iv * nu;
                    for (int iu = u0; iu <= u1; ++iu) {
                        const float4 r = __ldg(rk + row + iu);
                        const float w = hat_weight(fmaf(r.x, c0, r.y), j1f) *
                            hat_weight(fmaf(r.z, c0, r.w), j2f);
                        accv = fmaf(__ldg(vk + row + iu), w, accv);
                    }
                }
                acc[q] += static_cast<double>(accv);
            }
        }
    }
    const long plane = static_cast<long>(nx) * ny;
#pragma unroll
    for (int q = 0; q < ZV; ++q) {
        if (z0 + q >= nz) break;
        float* dst = vol + (z0 + q) * plane + static_cast<long>(y) * nx + x;
        *dst = accumulate ? static_cast<float>(*dst + acc[q]) : static_cast<float>(acc[q]);
    }
}

// ---------------------------------------------------------------------------
// Axial-column scans: every view has main axis x or y (so z is minor axis 2)
// and all rays of a detector column share their minor-1 parameters (a1, e1)
// bit for bit (the detector's v axis has no component along the main or
// minor-1 axis; checked on the device when the plan is built).  Their
// matched backprojection is joseph_bp_lines_kernel below.
// ---------------------------------------------------------------------------

// (a1, e1) of every detector column from its first row.
__global__ void joseph_column_table_kernel(const float4* __restrict__ rays, int n_views, int nu,
    int nv, float2* __restrict__ cols)
{
    const long n = static_cast<long>(n_views) * nu;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const long k = i / nu, iu = i - k * nu;
        const float4 r = rays[k * nu * nv + iu];
        cols[i] = make_float2(r.x, r.y);
    }
}

// flag[0] = 1 when some ray's (a1, e1) differs from its column's.
__global__ void joseph_column_check_kernel(const float4* __restrict__ rays,
    const float2* __restrict__ cols, int n_views, int nu, int nv, int* __restrict__ flag)
{
    const long n = static_cast<long>(n_views) * nu * nv;
    bool differs = false;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const long k = i / (static_cast<long>(nu) * nv);
        const long iu = i % nu;
        const float4 r = rays[i];
        const float2 c = cols[k * nu + iu];
        differs |= __float_as_uint(r.x) != __float_as_uint(c.x) ||
                   __float_as_uint(r.y) != __float_as_uint(c.y);
    }
    if (__any_sync(0xffffffffu, differs) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// ---------------------------------------------------------------------------
// Line backprojector (axial-column scans).  The transpose factors per
// detector column: voxel (s, j1, j2) of a view gets
//   sum over columns iu of h1(iu, s, j1) * L(iu, s, j2),
//   L(iu, s, j2) = sum over rows iv of t(iu, iv) h2(f2(iu, iv, s) - j2),
// where L, the column's rays splatted onto the z line of slice s, does not
// depend on j1.  A CTA owns 16 x 16 voxel columns of ZC slices.  Per view it
// builds, for each of its 16 slices, the lines of the detector columns that
// reach its 16 minor-1 indices (a warp per two adjacent slices, a lane per
// line, each lane walking its column's rays in order and splatting each
// onto both slices: every ray loaded once per two slices instead of once per
// voxel column it touches, about 2.5), then each thread adds the
// lines of its own column's candidate detector columns, weighted by h1, to
// its ZC sums.  Weights are the forward projector's; over sixteen views the sums
// are FP32 (lines in ray order, then over detector columns), then FP64 in
// shared memory.  Lines live in shared memory as [slice][slot][line], one
// bank per lane, slices 21 mod 32 words apart; a slice with more than
// kLineMax lines takes several passes.
// ---------------------------------------------------------------------------
constexpr int kLineBlock = 16;    // 16 x 16 voxel columns a CTA
constexpr int kLineThreads = 256;
constexpr int kLineMax = 32;      // lines of a slice per pass

// words from one slice's lines to the next: 21 mod 32.  A warp reads two
// slices (16 lanes each, similar detector columns) or sixteen slices (one
// lane each, similar column offsets); an odd shift near half the banks keeps
// both patterns apart (two slices: the second starts 21 banks on; sixteen:
// 21 s mod 32 are distinct)
template <int ZC>
__host__ __device__ constexpr int line_slice_words() { return (ZC + 2) * kLineMax + 21; }

template <int ZC>
constexpr size_t line_smem_bytes()
{
    return sizeof(double) * ZC * kLineThreads + sizeof(float) * kLineBlock * line_slice_words<ZC>() +
        sizeof(int4) * 2 * (kLineBlock + 1) + 16;
}

template <int ZC>
__global__ void __launch_bounds__(kLineThreads, 3) joseph_bp_lines_kernel(
    const float4* __restrict__ rays, const float* __restrict__ wv, const float2* __restrict__ cols,
    const ViewProj* __restrict__ vp, const JosephView* __restrict__ views, int n_views, int nu,
    int nv, int nx, int ny, int nz, float* __restrict__ vol, int accumulate)
{
    constexpr int B = kLineBlock, SL = ZC + 2, LM = kLineMax, PS = line_slice_words<ZC>();
    extern __shared__ __align__(16) unsigned char line_smem[];
    double* total = reinterpret_cast<double*>(line_smem);                 // [q][thread]
    float* lines = reinterpret_cast<float*>(total + ZC * kLineThreads);  // [slice][slot][line]
    // per view, by view parity: per slice u0, u1, v0, v1, then the passes.
    // A thread still reading view k's entries keeps them from being
    // overwritten (at view k + 2) until it reaches view k + 1's barrier, also
    // when view k needs no pass (and so no barrier of its own)
    int4* pbox2 = reinterpret_cast<int4*>(
        (reinterpret_cast<uintptr_t>(lines + B * PS) + 15) & ~static_cast<uintptr_t>(15));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tx = tid % B, ty = tid / B;
    const int X0 = blockIdx.x * B, Y0 = blockIdx.y * B, z0 = blockIdx.z * ZC;
    const int x = X0 + tx, y = Y0 + ty;
    const bool mine = x < nx && y < ny;
#pragma unroll
    for (int q = 0; q < ZC; ++q) total[q * kLineThreads + tid] = 0.0;
    // slot of floor(f2) + 1 from the rounding word of f2 - 1/2 (wrapping)
    const uint32_t slot0 = kMagicBits + static_cast<uint32_t>(z0 - 1);
    const f2 H = f2pack(0.5f, 0.5f), M = f2pack(kMagic, kMagic);
    float acc[ZC];  // FP32 over sixteen views, then into the FP64 sums
#pragma unroll
    for (int q = 0; q < ZC; ++q) acc[q] = 0.f;
    for (int k = 0; k < n_views; ++k) {
        const JosephView& j = views[k];
        const bool ax0 = j.axis == 0;
        const int S0 = ax0 ? X0 : Y0, J0 = ax0 ? Y0 : X0;  // first slice, first minor-1 index
        const int nS = min(B, j.n0 - S0), nJ = min(B, j.n1 - J0);
        int4* pbox = pbox2 + (k & 1) * (B + 1);
        int* pass_count = reinterpret_cast<int*>(pbox + B);
        const float half = 0.5f * (j.n0 - 1);
        if (tid < B) {
            int u0 = 0, u1 = -1, v0 = 0, v1 = -1;
            if (tid < nS)
                footprint_box_range(vp[k], j, static_cast<float>(S0 + tid) - half, J0,
                    J0 + nJ - 1, z0, z0 + ZC - 1, nu, nv, u0, u1, v0, v1);
            // slices 2i and 2i + 1 share the union of their boxes: a ray
            // outside a slice's own box adds nothing to the lines its voxel
            // columns read
            const bool some = u0 <= u1 && v0 <= v1;
            const int pu0 = __shfl_xor_sync(0xFFFFu, u0, 1), pu1 = __shfl_xor_sync(0xFFFFu, u1, 1);
            const int pv0 = __shfl_xor_sync(0xFFFFu, v0, 1), pv1 = __shfl_xor_sync(0xFFFFu, v1, 1);
            if (pu0 <= pu1 && pv0 <= pv1) {
                if (some) {
                    u0 = min(u0, pu0); u1 = max(u1, pu1);
                    v0 = min(v0, pv0); v1 = max(v1, pv1);
                } else {
                    u0 = pu0; u1 = pu1; v0 = pv0; v1 = pv1;
                }
            }
            pbox[tid] = make_int4(u0, u1, v0, v1);
            // passes of LM lines that the widest box needs
            int np = u0 <= u1 ? (u1 - u0 + LM) / LM : 0;
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) np = max(np, __shfl_xor_sync(0xFFFFu, np, o));
            if (tid == 0) *pass_count = np;
        }
        __syncthreads();
        const int passes = *pass_count;
        // this thread's voxel column: its slice, minor-1 index, candidates
        const int pl = ax0 ? tx : ty, j1 = ax0 ? y : x;
        const float c0 = static_cast<float>(S0 + pl) - half;
        int cu0 = 0, cu1 = -1, cv0, cv1;
        if (mine) footprint_box(vp[k], j, c0, j1, z0, z0 + ZC - 1, nu, nv, cu0, cu1, cv0, cv1);
        const float j1f = static_cast<float>(j1);
        const float2* ck = cols + static_cast<long>(k) * nu;
        for (int pass = 0; pass < passes; ++pass) {
            // ---- lines: warp w builds slices 2w and 2w + 1, lane = line
            {
                static_assert(B == 2 * (kLineThreads / 32), "a warp per two slices");
                const int sp = 2 * warp;
                const int4 b = pbox[sp];  // the pair's box
                float* La = lines + sp * PS + lane;
                float* Lb = La + PS;
#pragma unroll
                // slots 1 .. ZC are read; the end slots (z0 - 1, z0 + ZC) only
                // take the far halves of splats and are never read, so they
                // are not cleared
                for (int q = 1; q <= ZC; ++q) {
                    La[q * LM] = 0.f;
                    Lb[q * LM] = 0.f;
                }
                const int iu = b.x + pass * LM + lane;
                if (iu <= b.y) {
                    const float csa = static_cast<float>(S0 + sp) - half;
                    const float csb = static_cast<float>(S0 + sp + 1) - half;
                    const long r0 = (static_cast<long>(k) * nv + b.z) * nu + iu;
                    // (a2, e2) are the last two floats of each ray's record
                    const float2* ae = reinterpret_cast<const float2*>(rays) + 2 * r0 + 1;
                    const float* tv = wv + r0;
                    const long st = 2l * nu;  // float2 records from one row to the next
                    int iv = b.z;
                    auto splat = [&](const float2 a, const float v) {
                        const f2 f = f2pack(fmaf(a.x, csa, a.y), fmaf(a.x, csb, a.y));
                        const f2 t = f2add(f2sub(f, H), M);
                        float ta, tb, wa, wb;
                        f2unpack(t, ta, tb);
                        f2unpack(f2sub(f, f2sub(t, M)), wa, wb);
                        const uint32_t sa = __float_as_uint(ta) - slot0, sb = __float_as_uint(tb) - slot0;
                        if (sa <= static_cast<uint32_t>(ZC)) {
                            float* o = La + sa * LM;
                            o[0] = fmaf(v, 1.f - wa, o[0]);
                            o[LM] = fmaf(v, wa, o[LM]);
                        }
                        if (sb <= static_cast<uint32_t>(ZC)) {
                            float* o = Lb + sb * LM;
                            o[0] = fmaf(v, 1.f - wb, o[0]);
                            o[LM] = fmaf(v, wb, o[LM]);
                        }
                    };
                    // eight rays per step: their loads are in flight together
                    for (; iv + 7 <= b.w; iv += 8, ae += 8 * st, tv += 8 * nu) {
                        float2 a[8];
                        float v[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            a[i] = __ldg(ae + i * st);
                            v[i] = __ldg(tv + i * nu);
                        }
#pragma unroll
                        for (int i = 0; i < 8; ++i) splat(a[i], v[i]);
                    }
                    for (; iv <= b.w; ++iv, ae += st, tv += nu) splat(__ldg(ae), __ldg(tv));
                }
            }
            __syncthreads();
            // ---- this column: its candidates among this pass's lines
            if (mine) {
                const int base = pbox[pl].x + pass * LM;
                const int lo = max(cu0, base), hi = min(min(cu1, pbox[pl].y), base + LM - 1);
                const float* Lp = lines + pl * PS - base;
                for (int iu = lo; iu <= hi; ++iu) {
                    // the forward projector's minor-1 weights
                    const float2 ce = __ldg(ck + iu);
                    const float f1 = fmaf(ce.x, c0, ce.y);
                    const float fl1 = floorf(f1);
                    const float w1 = f1 - fl1;
                    const float h1 = fl1 == j1f ? 1.f - w1 : (fl1 + 1.f == j1f ? w1 : 0.f);
                    if (h1 == 0.f) continue;
#pragma unroll
                    for (int q = 0; q < ZC; ++q) acc[q] = fmaf(h1, Lp[(q + 1) * LM + iu], acc[q]);
                }
            }
            __syncthreads();
        }
        if ((k & 15) == 15 || k + 1 == n_views) {
#pragma unroll
            for (int q = 0; q < ZC; ++q) {
                total[q * kLineThreads + tid] += static_cast<double>(acc[q]);
                acc[q] = 0.f;
            }
        }
    }
    if (!mine) return;
    const long plane = static_cast<long>(nx) * ny;
#pragma unroll
    for (int q = 0; q < ZC; ++q) {
        if (z0 + q >= nz) break;
        float* dst = vol + (z0 + q) * plane + static_cast<long>(y) * nx + x;
        const double a = total[q * kLineThreads + tid];
        *dst = accumulate ? static_cast<float>(*dst + a) : static_cast<float>(a);
    }
}

} // namespace

cudaError_t launch_joseph_column_table(const float4* rays, int n_views, int nu, int nv,
    float2* cols, int* flag, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    joseph_column_table_kernel<<<148 * 4, 256, 0, s>>>(rays, n_views, nu, nv, cols);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    joseph_column_check_kernel<<<148 * 8, 256, 0, s>>>(rays, cols, n_views, nu, nv, flag);
    return cudaGetLastError();
}

cudaError_t launch_joseph_bp_lines(const float* proj, const float4* rays, const float* lens,
    const float2* cols, const float* view_proj, const JosephView* views, int n_views, int nu,
    int nv, const ykb_volume& vol, float* weighted, float* out, int accumulate, cudaStream_t s)
{
    const long n = static_cast<long>(n_views) * nu * nv;
    joseph_weight_rays_kernel<<<148 * 8, 256, 0, s>>>(proj, lens, n, weighted);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    constexpr int ZC = 16;
    auto k = joseph_bp_lines_kernel<ZC>;
    constexpr size_t smem = line_smem_bytes<ZC>();
    if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
             static_cast<int>(smem))) != cudaSuccess)
        return e;
    const dim3 grid((vol.nx + kLineBlock - 1) / kLineBlock, (vol.ny + kLineBlock - 1) / kLineBlock,
        (vol.nz + ZC - 1) / ZC);
    k<<<grid, kLineThreads, smem, s>>>(rays, weighted, cols, reinterpret_cast<const ViewProj*>(view_proj),
        views, n_views, nu, nv, vol.nx, vol.ny, vol.nz, out, accumulate);
    return cudaGetLastError();
}

cudaError_t launch_joseph_transpose(const float* vol, int nx, int ny, int nz, float* vol_yzx,
    float* vol_xzy, cudaStream_t s)
{
    if (vol_yzx) {
        const dim3 grid((nx + 127) / 128, ny, nz);
        transpose_yzx_kernel<<<grid, 128, 0, s>>>(vol, nx, ny, nz, vol_yzx);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (vol_xzy) {
        const dim3 grid((nx + 31) / 32, (ny + 31) / 32, nz);
        transpose_xzy_kernel<<<grid, dim3(32, 8), 0, s>>>(vol, nx, ny, nz, vol_xzy);
    }
    return cudaGetLastError();
}

cudaError_t launch_joseph_fp(const float* slabs[3], const JosephView* views,
    const int* view_axis_host, int n_views, int nu, int nv, float* proj, int accumulate,
    cudaStream_t s)
{
    // consecutive views with the same main axis share one launch (the
    // forEachAxisRun grouping of YkOperatorKernelTypes.cuh:171-210)
    int first = 0;
    while (first < n_views) {
        const int axis = view_axis_host[first];
        int end = first + 1;
        while (end < n_views && view_axis_host[end] == axis) ++end;
        int done = first;
        while (done < end) {
            const int count = min(end - done, 65535);
            const dim3 grid((nu + 31) / 32, (nv + 3) / 4, count);
            if (axis == 2)
                joseph_fp_kernel<<<grid, dim3(32, 4), 0, s>>>(slabs[axis], views, done, nu, nv,
                    proj, accumulate);
            else
                joseph_fp_padded_kernel<<<grid, dim3(32, 4), 0, s>>>(slabs[axis], views, done, nu,
                    nv, proj, accumulate);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            done += count;
        }
        first = end;
    }
    return cudaSuccess;
}

cudaError_t launch_joseph_ray_table(const JosephView* views, int n_views, int nu, int nv,
    float4* rays, float* lens, cudaStream_t s)
{
    for (int done = 0; done < n_views; done += 65535) {
        const int count = min(n_views - done, 65535);
        const dim3 grid((nu + 31) / 32, (nv + 3) / 4, count);
        joseph_ray_table_kernel<<<grid, dim3(32, 4), 0, s>>>(views + done, nu, nv,
            rays + static_cast<long>(done) * nu * nv, lens + static_cast<long>(done) * nu * nv);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_joseph_bp(const float* proj, const float4* rays, const float* lens,
    const float* view_proj, const JosephView* views, int n_views, int nu, int nv,
    const ykb_volume& vol, float* weighted, float* out, int accumulate, cudaStream_t s)
{
    const long n = static_cast<long>(n_views) * nu * nv;
    joseph_weight_rays_kernel<<<148 * 8, 256, 0, s>>>(proj, lens, n, weighted);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    constexpr int ZV = 4;
    const dim3 grid((vol.nx + 31) / 32, (vol.ny + 7) / 8, (vol.nz + ZV - 1) / ZV);
    joseph_bp_kernel<ZV><<<grid, dim3(32, 8), 0, s>>>(weighted, rays,
        reinterpret_cast<const ViewProj*>(view_proj), views, n_views, nu, nv, vol.nx, vol.ny,
        vol.nz, out, accumulate);
    return cudaGetLastError();
}

} // namespace ykb
