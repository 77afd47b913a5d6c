// FDK kernels for sm_100a: cosine preweight, FP32 Toeplitz ramp filter and
// voxel-driven weighted backprojection.
#include "ykb_internal.hpp"
#include "pseudo_weight.cuh"

#include <cuda_bf16.h>

namespace ykb {
namespace {

template <typename T> __device__ __forceinline__ float load_as_float(const T* p);
template <> __device__ __forceinline__ float load_as_float<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float load_as_float<__nv_bfloat16>(const __nv_bfloat16* p)
{
    return __bfloat162float(*p);
}

// Cosine preweight of .../FDK/kernels/YkFDKPreWeightKernels.cu:374-402:
// out = in * DSD/|q(u,v)| * DSD/(2 DSO), q = detS + u detU + v detV - src,
// with samples the padded FFT row would drop set to zero.  FP64 geometry,
// 1/|q| by an FP32 rsqrt refined with one FP64 Newton step.
template <typename TIn>
__global__ void __launch_bounds__(128) preweight_kernel(const TIn* __restrict__ in,
    const FdkPreweightView* __restrict__ pw, const float* __restrict__ parker, int nu, int nv,
    float* __restrict__ out)
{
    const long row = blockIdx.x;
    const int view = static_cast<int>(row / nv);
    const int iv = static_cast<int>(row - static_cast<long>(view) * nv);
    const FdkPreweightView& p = pw[view];
    const double qx0 = p.detS[0] + iv * p.detV[0] - p.src[0];
    const double qy0 = p.detS[1] + iv * p.detV[1] - p.src[1];
    const double qz0 = p.detS[2] + iv * p.detV[2] - p.src[2];
    const double scale = p.dsd * p.wgeom;
    const TIn* src = in + row * nu;
    float* dst = out + row * nu;
    for (int iu = threadIdx.x; iu < nu; iu += blockDim.x) {
        const double qx = fma(static_cast<double>(iu), p.detU[0], qx0);
        const double qy = fma(static_cast<double>(iu), p.detU[1], qy0);
        const double qz = fma(static_cast<double>(iu), p.detU[2], qz0);
        const double r2 = fmax(qx * qx + qy * qy + qz * qz, 1e-20);
        double r = rsqrtf(static_cast<float>(r2));
        r = r * (1.5 - 0.5 * r2 * r * r);
        const bool placed = iu >= p.in_lo && iu < p.in_hi;
        float wt = static_cast<float>(scale * r);
        if (parker) wt *= parker[static_cast<long>(view) * nu + iu];
        dst[iu] = placed ? load_as_float(src + iu) * wt : 0.f;
    }
}

// Ramp filter as a Toeplitz product C[m][j] = sum_k A[m][k] h[j-k] over all
// rows m = (view, v): the linear form of the reference's pad -> R2C -> x w ->
// C2R -> crop (.../FDK/kernels/YkFDKFilterKernels.cu:32-140).  FP32 SIMT
// GEMM, 64x128 output tile per block, 4x8 per thread.  The Toeplitz operand
// is never materialised: a thread keeps the BK+7 lags its 8 columns need
// for a k-tile in registers.
constexpr int RBM = 64, RBN = 128, RBK = 32;

template <bool PAIR>
__global__ void __launch_bounds__(256) ramp_fp32_kernel(const float* __restrict__ A,
    const float* __restrict__ h, const FdkPreweightView* __restrict__ pwv, long rows,
    int nu, int nv, float* __restrict__ C, int ldc)
{
    __shared__ __align__(16) float As[RBK][RBM + 4];
    __shared__ float hs[RBN + RBK];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const long m0 = static_cast<long>(blockIdx.y) * RBM;
    const int j0 = blockIdx.x * RBN;
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[i][q] = 0.f;

    for (int k0 = 0; k0 < nu; k0 += RBK) {
        // A tile: warp w loads rows w, w+8, ...; lane = k offset (coalesced)
        {
            const int kk = tid & 31;
            const int rbase = tid >> 5;
#pragma unroll
            for (int i = 0; i < RBM / 8; ++i) {
                const int r = rbase + 8 * i;
                const long m = m0 + r;
                const int k = k0 + kk;
                As[kk][r] = (m < rows && k < nu) ? __ldg(A + m * nu + k) : 0.f;
            }
        }
        // lags d = j - k for j in [j0, j0+RBN), k in [k0, k0+RBK)
        for (int i = tid; i < RBN + RBK - 1; i += 256) {
            const int d = j0 - k0 - (RBK - 1) + i;
            hs[i] = (d > -nu && d < nu) ? __ldg(h + d + nu - 1) : 0.f;
        }
        __syncthreads();
        float hr[RBK + 7];
#pragma unroll
        for (int i = 0; i < RBK + 7; ++i) hr[i] = hs[tx * 8 + i];
#pragma unroll
        for (int kk = 0; kk < RBK; ++kk) {
            const float4 a = *reinterpret_cast<const float4*>(&As[kk][ty * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float b = hr[q - kk + RBK - 1];
#pragma unroll
                for (int i = 0; i < 4; ++i) acc[i][q] = fmaf(av[i], b, acc[i][q]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const long m = m0 + ty * 4 + i;
        if (m >= rows) continue;
        const FdkPreweightView& p = pwv[m / nv];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int j = j0 + tx * 8 + q;
            if (j >= nu) continue;
            const float v = (j >= p.out_lo && j < p.out_hi) ? acc[i][q] : 0.f;
            if constexpr (!PAIR) {
                C[m * ldc + j] = v;
            } else {
                // tap pairs: left of pair j, right of pair j-1; the pairs
                // around the row are zero where they reach outside it
                float* row = C + m * 2 * ldc + 2 * kPairLead;
                row[2 * j] = v;
                row[2 * j - 1] = v;
                if (j == 0) row[-2] = row[-3] = row[-4] = 0.f;
                if (j == nu - 1) row[2 * j + 1] = 0.f;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Voxel-driven weighted backprojection:
//   vol(P) += sum_views bilinear_view(u, v) * SID^2 dtheta (2pi/range) / depth^2
// with u = cu.P/cd.P, v = cv.P/cd.P, depth = cr.P (the arithmetic of
// fdk_bp_kernel, .../FDK/kernels/YkFDKBpKernels.cu:112-209, with exact
// software bilinear weights and zero outside the detector instead of the
// 8-bit hardware texture filter).  One thread owns ZT consecutive voxels of
// a z-column and accumulates all views in registers; a block covers 32x8
// columns.
// AXIAL: u, cd.P and cr.P do not depend on z (untilted detector on a
// circular orbit); the per-column terms are evaluated once per view in FP64
// and only v advances along the column.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ float tap(const T* img, int nu, int nv, int ld, int iu, int iv)
{
    return (static_cast<unsigned>(iu) < static_cast<unsigned>(nu) &&
            static_cast<unsigned>(iv) < static_cast<unsigned>(nv))
        ? load_as_float(img + static_cast<long>(iv) * ld + iu) : 0.f;
}

__device__ __forceinline__ double rcp_fp64(double x)
{
    double r = static_cast<double>(__frcp_rn(static_cast<float>(x)));
    r = r * (2.0 - x * r);
    r = r * (2.0 - x * r);
    return r;
}

template <int ZT, bool AXIAL, typename T>
__global__ void __launch_bounds__(256) fdk_bp_kernel(const T* __restrict__ proj,
    const FdkViewCoef* __restrict__ coef, int n_views, int nu, int nv, int ld, VolumeGrid g,
    float* __restrict__ vol, int accumulate)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * ZT;
    if (x >= g.nx || y >= g.ny) return;
    const double X = g.ox + x * g.vx;
    const double Y = g.oy + y * g.vy;
    const double Z0 = g.oz + z0 * g.vz;
    float acc[ZT];
#pragma unroll
    for (int i = 0; i < ZT; ++i) acc[i] = 0.f;
    const long view_elems = static_cast<long>(ld) * nv;

    for (int k = 0; k < n_views; ++k) {
        const FdkViewCoef& c = coef[k];
        const T* img = proj + k * view_elems;
        if constexpr (AXIAL) {
            const double den = fma(c.cd[1], Y, fma(c.cd[0], X, c.cd[3]));
            const double rd = rcp_fp64(den);
            const double un = fma(c.cu[1], Y, fma(c.cu[0], X, c.cu[3]));
            const double vn = fma(c.cv[2], Z0, fma(c.cv[1], Y, fma(c.cv[0], X, c.cv[3])));
            const double dep = fma(c.cr[1], Y, fma(c.cr[0], X, c.cr[3]));
            const float u = static_cast<float>(un * rd);
            const float vb = static_cast<float>(vn * rd);
            const float vs = static_cast<float>(c.cv[2] * g.vz * rd);
            const float w = static_cast<float>(c.wbase / (dep * dep));
            const float fu = floorf(u);
            const int iu = static_cast<int>(fu);
            const float au = u - fu;
#pragma unroll
            for (int i = 0; i < ZT; ++i) {
                const float v = fmaf(static_cast<float>(i), vs, vb);
                const float fv = floorf(v);
                const int iv = static_cast<int>(fv);
                const float av = v - fv;
                const float p00 = tap(img, nu, nv, ld, iu, iv), p10 = tap(img, nu, nv, ld, iu + 1, iv);
                const float p01 = tap(img, nu, nv, ld, iu, iv + 1), p11 = tap(img, nu, nv, ld, iu + 1, iv + 1);
                const float r0 = fmaf(au, p10 - p00, p00);
                const float r1 = fmaf(au, p11 - p01, p01);
                acc[i] = fmaf(w, fmaf(av, r1 - r0, r0), acc[i]);
            }
        } else {
            const double den0 = fma(c.cd[2], Z0, fma(c.cd[1], Y, fma(c.cd[0], X, c.cd[3])));
            const double un0 = fma(c.cu[2], Z0, fma(c.cu[1], Y, fma(c.cu[0], X, c.cu[3])));
            const double vn0 = fma(c.cv[2], Z0, fma(c.cv[1], Y, fma(c.cv[0], X, c.cv[3])));
            const double dp0 = fma(c.cr[2], Z0, fma(c.cr[1], Y, fma(c.cr[0], X, c.cr[3])));
            const float s = static_cast<float>(c.wbase);
            // per-column base values in FP64 rounded once; z increments in FP32
            const float dn = static_cast<float>(den0), ddn = static_cast<float>(c.cd[2] * g.vz);
            const float uu = static_cast<float>(un0), dun = static_cast<float>(c.cu[2] * g.vz);
            const float vv = static_cast<float>(vn0), dvn = static_cast<float>(c.cv[2] * g.vz);
            const float dp = static_cast<float>(dp0), ddp = static_cast<float>(c.cr[2] * g.vz);
#pragma unroll
            for (int i = 0; i < ZT; ++i) {
                const float fi = static_cast<float>(i);
                const float rden = 1.f / fmaf(fi, ddn, dn);
                const float u = fmaf(fi, dun, uu) * rden;
                const float v = fmaf(fi, dvn, vv) * rden;
                const float rdep = 1.f / fmaf(fi, ddp, dp);
                const float w = s * rdep * rdep;
                const float fu = floorf(u), fv = floorf(v);
                const int iu = static_cast<int>(fu), iv = static_cast<int>(fv);
                const float au = u - fu, av = v - fv;
                const float p00 = tap(img, nu, nv, ld, iu, iv), p10 = tap(img, nu, nv, ld, iu + 1, iv);
                const float p01 = tap(img, nu, nv, ld, iu, iv + 1), p11 = tap(img, nu, nv, ld, iu + 1, iv + 1);
                const float r0 = fmaf(au, p10 - p00, p00);
                const float r1 = fmaf(au, p11 - p01, p01);
                acc[i] = fmaf(w, fmaf(av, r1 - r0, r0), acc[i]);
            }
        }
    }
    const long plane = static_cast<long>(g.nx) * g.ny;
#pragma unroll
    for (int i = 0; i < ZT; ++i) {
        const int z = z0 + i;
        if (z >= g.nz) break;
        float* dst = vol + z * plane + static_cast<long>(y) * g.nx + x;
        *dst = accumulate ? *dst + acc[i] : acc[i];
    }
}

// Pseudo-matched backprojection with bounds-checked loads: the non-axial
// column walk of fdk_bp_kernel with the weight of pseudo_weight.cuh.
template <int ZT>
__global__ void __launch_bounds__(256) pseudo_bp_kernel(const float* __restrict__ proj,
    const FdkViewCoef* __restrict__ coef, const PseudoViewCoef* __restrict__ pseudo, int n_views,
    int nu, int nv, VolumeGrid g, float* __restrict__ vol, int accumulate)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * ZT;
    if (x >= g.nx || y >= g.ny) return;
    const double X = g.ox + x * g.vx;
    const double Y = g.oy + y * g.vy;
    const double Z0 = g.oz + z0 * g.vz;
    float acc[ZT];
#pragma unroll
    for (int i = 0; i < ZT; ++i) acc[i] = 0.f;
    const long view_elems = static_cast<long>(nu) * nv;
    for (int k = 0; k < n_views; ++k) {
        const FdkViewCoef& c = coef[k];
        const PseudoViewCoef& p = pseudo[k];
        const float* img = proj + k * view_elems;
        const double den0 = fma(c.cd[2], Z0, fma(c.cd[1], Y, fma(c.cd[0], X, c.cd[3])));
        const double un0 = fma(c.cu[2], Z0, fma(c.cu[1], Y, fma(c.cu[0], X, c.cu[3])));
        const double vn0 = fma(c.cv[2], Z0, fma(c.cv[1], Y, fma(c.cv[0], X, c.cv[3])));
        const float dn = static_cast<float>(den0), ddn = static_cast<float>(c.cd[2] * g.vz);
        const float uu = static_cast<float>(un0), dun = static_cast<float>(c.cu[2] * g.vz);
        const float vv = static_cast<float>(vn0), dvn = static_cast<float>(c.cv[2] * g.vz);
        const PseudoColumn col = pseudo_column(p, X, Y, Z0, g.vz);
#pragma unroll
        for (int i = 0; i < ZT; ++i) {
            const float fi = static_cast<float>(i);
            const float den = fmaf(fi, ddn, dn);
            if (!(den > 1e-8f)) continue;  // the voxel is not in front of the source
            const float rden = 1.f / den;
            const float u = fmaf(fi, dun, uu) * rden;
            const float v = fmaf(fi, dvn, vv) * rden;
            if (!(fabsf(u) < 1e7f && fabsf(v) < 1e7f)) continue;
            const float w = pseudo_weight(p, col, fi, u, v);
            const float fu = floorf(u), fv = floorf(v);
            const int iu = static_cast<int>(fu), iv = static_cast<int>(fv);
            const float au = u - fu, av = v - fv;
            const float p00 = tap(img, nu, nv, nu, iu, iv), p10 = tap(img, nu, nv, nu, iu + 1, iv);
            const float p01 = tap(img, nu, nv, nu, iu, iv + 1), p11 = tap(img, nu, nv, nu, iu + 1, iv + 1);
            const float r0 = fmaf(au, p10 - p00, p00);
            const float r1 = fmaf(au, p11 - p01, p01);
            acc[i] = fmaf(w, fmaf(av, r1 - r0, r0), acc[i]);
        }
    }
    const long plane = static_cast<long>(g.nx) * g.ny;
#pragma unroll
    for (int i = 0; i < ZT; ++i) {
        const int z = z0 + i;
        if (z >= g.nz) break;
        float* dst = vol + z * plane + static_cast<long>(y) * g.nx + x;
        *dst = accumulate ? *dst + acc[i] : acc[i];
    }
}

} // namespace

cudaError_t launch_pseudo_backproject(const float* proj, const FdkViewCoef* coef,
    const PseudoViewCoef* pseudo, int n_views, int nu, int nv, const VolumeGrid& grid,
    float* vol, int accumulate, cudaStream_t s)
{
    constexpr int ZT = 8;
    const dim3 blocks((grid.nx + 31) / 32, (grid.ny + 7) / 8, (grid.nz + ZT - 1) / ZT);
    pseudo_bp_kernel<ZT><<<blocks, dim3(32, 8), 0, s>>>(proj, coef, pseudo, n_views, nu, nv,
        grid, vol, accumulate);
    return cudaGetLastError();
}

cudaError_t launch_fdk_preweight(const void* proj, int proj_dtype,
    const FdkPreweightView* pw, const float* parker, int n_views, int nu, int nv, float* out,
    cudaStream_t s)
{
    const long rows = static_cast<long>(n_views) * nv;
    if (rows <= 0) return cudaSuccess;
    if (proj_dtype == YKB_DTYPE_BF16)
        preweight_kernel<__nv_bfloat16><<<static_cast<unsigned>(rows), 128, 0, s>>>(
            static_cast<const __nv_bfloat16*>(proj), pw, parker, nu, nv, out);
    else
        preweight_kernel<float><<<static_cast<unsigned>(rows), 128, 0, s>>>(
            static_cast<const float*>(proj), pw, parker, nu, nv, out);
    return cudaGetLastError();
}

cudaError_t launch_fdk_ramp_fp32(const float* pw_rows, const float* h_dev,
    const FdkPreweightView* pwv, int n_views, int nu, int nv, float* out, int layout,
    int ldc, cudaStream_t s)
{
    const long rows = static_cast<long>(n_views) * nv;
    if (rows <= 0) return cudaSuccess;
    const dim3 grid((nu + RBN - 1) / RBN, static_cast<unsigned>((rows + RBM - 1) / RBM));
    if (layout == kFilteredPairs)
        ramp_fp32_kernel<true><<<grid, 256, 0, s>>>(pw_rows, h_dev, pwv, rows, nu, nv, out, ldc);
    else
        ramp_fp32_kernel<false><<<grid, 256, 0, s>>>(pw_rows, h_dev, pwv, rows, nu, nv, out, ldc);
    return cudaGetLastError();
}

cudaError_t launch_fdk_backproject(const void* filtered, int dtype, const FdkViewCoef* coef,
    int n_views, int nu, int nv, int ld, const VolumeGrid& g, bool axial, float* vol,
    int accumulate, cudaStream_t s)
{
    constexpr int ZT = 16;
    const dim3 block(32, 8);
    const dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + ZT - 1) / ZT);
    if (dtype == YKB_DTYPE_BF16) {
        auto p = static_cast<const __nv_bfloat16*>(filtered);
        if (axial) fdk_bp_kernel<ZT, true><<<grid, block, 0, s>>>(p, coef, n_views, nu, nv, ld, g, vol, accumulate);
        else fdk_bp_kernel<ZT, false><<<grid, block, 0, s>>>(p, coef, n_views, nu, nv, ld, g, vol, accumulate);
    } else {
        auto p = static_cast<const float*>(filtered);
        if (axial) fdk_bp_kernel<ZT, true><<<grid, block, 0, s>>>(p, coef, n_views, nu, nv, ld, g, vol, accumulate);
        else fdk_bp_kernel<ZT, false><<<grid, block, 0, s>>>(p, coef, n_views, nu, nv, ld, g, vol, accumulate);
    }
    return cudaGetLastError();
}

} // namespace ykb
