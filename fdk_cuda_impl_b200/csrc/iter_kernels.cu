// Vector kernels of the iterative solvers that consume the projector pair
// (CGLS of src/Reconstruction/Iterative/Flat/YkCglsBackends.hpp:70-150 over
// the reductions of src/Reconstruction/Iterative/Common/kernels/
// YkIterKernels.cu:367-430).
//
// The reference reduces its dot products in FP32 and copies the partial sums
// to the host on every call, synchronising the stream.  Here:
//   * dot_f64: FP64 accumulation of FP32 products, 16-byte loads, a fixed
//     grid of 4 x 148 blocks whose FP64 partials a second one-block kernel
//     sums in a fixed order: deterministic, and the result stays on the
//     device;
//   * the CGLS vector updates read their step sizes (ratios of those FP64
//     sums) from device memory, so a CGLS iteration never waits on the host.
// All kernels are HBM-bound streams.
#include "ykb_internal.hpp"

namespace ykb {
namespace {

constexpr int kDotBlocks = 4 * 148;
constexpr int kDotThreads = 256;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block sum of v into out (thread 0); blockDim.x == kDotThreads
__device__ __forceinline__ void block_sum(double v, double* out)
{
    __shared__ double warps[kDotThreads / 32];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) warps[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < kDotThreads / 32 ? warps[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) *out = v;
    }
}

__global__ void __launch_bounds__(kDotThreads) dot_partials_kernel(const float* __restrict__ a,
    const float* __restrict__ b, size_t n, double* __restrict__ partials)
{
    double acc = 0.0;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    const size_t tid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool vec = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) == 0;
    size_t done = 0;
    if (vec) {
        const size_t n4 = n / 4;
        const float4* a4 = reinterpret_cast<const float4*>(a);
        const float4* b4 = reinterpret_cast<const float4*>(b);
        for (size_t i = tid; i < n4; i += stride) {
            const float4 x = __ldg(a4 + i), y = __ldg(b4 + i);
            acc += static_cast<double>(x.x) * y.x + static_cast<double>(x.y) * y.y +
                static_cast<double>(x.z) * y.z + static_cast<double>(x.w) * y.w;
        }
        done = n4 * 4;
    }
    for (size_t i = done + tid; i < n; i += stride)
        acc += static_cast<double>(__ldg(a + i)) * __ldg(b + i);
    block_sum(acc, partials + blockIdx.x);
}

__global__ void __launch_bounds__(kDotThreads) sum_partials_kernel(const double* __restrict__ partials,
    int count, double* __restrict__ result)
{
    double acc = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partials[i];
    block_sum(acc, result);
}

__device__ __forceinline__ float safe_ratio(const double* num, const double* den)
{
    const double d = *den;
    return d > 1e-300 ? static_cast<float>(*num / d) : 0.f;
}

// x += alpha p, r -= alpha w, alpha = gamma / ww
__global__ void cgls_xr_kernel(const double* __restrict__ gamma, const double* __restrict__ ww,
    float* __restrict__ x, const float* __restrict__ p, size_t nx, float* __restrict__ r,
    const float* __restrict__ w, size_t nr)
{
    const float alpha = safe_ratio(gamma, ww);
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nx + nr;
         i += stride) {
        if (i < nx) x[i] = fmaf(alpha, p[i], x[i]);
        else r[i - nx] = fmaf(-alpha, w[i - nx], r[i - nx]);
    }
}

// p = z + beta p, beta = gamma_new / gamma_old
__global__ void cgls_p_kernel(const double* __restrict__ gamma_new,
    const double* __restrict__ gamma_old, float* __restrict__ p, const float* __restrict__ z,
    size_t n)
{
    const float beta = safe_ratio(gamma_new, gamma_old);
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        p[i] = fmaf(beta, p[i], z[i]);
}

} // namespace

int dot_partial_count() { return kDotBlocks; }

cudaError_t launch_dot_f64(const float* a, const float* b, size_t n, double* partials,
    double* result, cudaStream_t s)
{
    dot_partials_kernel<<<kDotBlocks, kDotThreads, 0, s>>>(a, b, n, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    sum_partials_kernel<<<1, kDotThreads, 0, s>>>(partials, kDotBlocks, result);
    return cudaGetLastError();
}

cudaError_t launch_cgls_xr(const double* gamma, const double* ww, float* x, const float* p,
    size_t nx, float* r, const float* w, size_t nr, cudaStream_t s)
{
    cgls_xr_kernel<<<148 * 8, 256, 0, s>>>(gamma, ww, x, p, nx, r, w, nr);
    return cudaGetLastError();
}

cudaError_t launch_cgls_p(const double* gamma_new, const double* gamma_old, float* p,
    const float* z, size_t n, cudaStream_t s)
{
    cgls_p_kernel<<<148 * 8, 256, 0, s>>>(gamma_new, gamma_old, p, z, n);
    return cudaGetLastError();
}

} // namespace ykb
