// Shared-memory load bandwidth of this GPU, measured: the on-chip peak that
// the FDK backprojection (two 8-byte shared loads of bilinear tap pairs per
// voxel update) is reported against.
//
// Every CTA fills 16 KB of shared memory and its 256 threads stream it back
// with vector loads: lane i reads the WORDS 32-bit words at word offset
// WORDS * i of a row of 256 * WORDS words, so the 32 lanes of a warp cover
// consecutive banks (no conflicts).  The loaded words are XOR-folded into
// registers that a never-taken store keeps
// alive; volatile shared loads are never hoisted out of the loop or merged
// (the loaded words do not change, so plain loads would be).  Four CTAs per
// SM keep enough warps in flight to saturate the pipe.
#include "ykb_internal.hpp"

#include <algorithm>

namespace ykb {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeRows = 4;  // 16 KB for 16-byte loads

__device__ __forceinline__ uint32_t probe_smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <int WORDS, int OFF>
__device__ __forceinline__ void probe_load(uint32_t addr, uint32_t& a, uint32_t& b)
{
    if constexpr (WORDS == 2) {
        uint32_t x, y;
        asm volatile("ld.volatile.shared.v2.u32 {%0, %1}, [%2+%3];" : "=r"(x), "=r"(y) : "r"(addr), "n"(OFF));
        a ^= x; b ^= y;
    } else {
        uint32_t x, y, z, w;
        asm volatile("ld.volatile.shared.v4.u32 {%0, %1, %2, %3}, [%4+%5];"
            : "=r"(x), "=r"(y), "=r"(z), "=r"(w) : "r"(addr), "n"(OFF));
        a ^= x ^ z; b ^= y ^ w;
    }
}

template <int WORDS>
__global__ void __launch_bounds__(kProbeThreads) shared_load_kernel(int iters, uint32_t* sink)
{
    __shared__ __align__(16) uint32_t buf[kProbeRows * kProbeThreads * 4];
    for (int i = threadIdx.x; i < kProbeRows * kProbeThreads * 4; i += kProbeThreads)
        buf[i] = 2654435761u * static_cast<uint32_t>(i + 1);
    __syncthreads();
    constexpr int ROW = kProbeThreads * WORDS * 4;  // bytes of one row
    const uint32_t addr = probe_smem_addr(buf) + threadIdx.x * WORDS * 4;
    uint32_t a0 = 0, b0 = 0, a1 = 0, b1 = 0;
    for (int it = 0; it < iters; ++it) {
        // 16 loads per iteration, two independent XOR chains
        probe_load<WORDS, 0 * ROW>(addr, a0, b0);
        probe_load<WORDS, 1 * ROW>(addr, a1, b1);
        probe_load<WORDS, 2 * ROW>(addr, a0, b0);
        probe_load<WORDS, 3 * ROW>(addr, a1, b1);
        probe_load<WORDS, 0 * ROW>(addr, a0, b0);
        probe_load<WORDS, 1 * ROW>(addr, a1, b1);
        probe_load<WORDS, 2 * ROW>(addr, a0, b0);
        probe_load<WORDS, 3 * ROW>(addr, a1, b1);
        probe_load<WORDS, 0 * ROW>(addr, a0, b0);
        probe_load<WORDS, 1 * ROW>(addr, a1, b1);
        probe_load<WORDS, 2 * ROW>(addr, a0, b0);
        probe_load<WORDS, 3 * ROW>(addr, a1, b1);
        probe_load<WORDS, 0 * ROW>(addr, a0, b0);
        probe_load<WORDS, 1 * ROW>(addr, a1, b1);
        probe_load<WORDS, 2 * ROW>(addr, a0, b0);
        probe_load<WORDS, 3 * ROW>(addr, a1, b1);
    }
    const uint32_t r = a0 ^ b0 ^ a1 ^ b1;
    if (r == 0x9e3779b9u) sink[0] = r;  // keeps the folds alive; harmless if taken
}

} // namespace
} // namespace ykb

using namespace ykb;

extern "C" YKB_API ykb_status ykb_measure_shared_load_gbs(int device, int bytes_per_lane,
    double* gbs)
{
    clear_error();
    if (!gbs) return (set_error("null output"), YKB_ERR_INVALID_BUFFER);
    if (bytes_per_lane != 8 && bytes_per_lane != 16)
        return (set_error("bytes_per_lane must be 8 or 16"), YKB_ERR_INVALID_CONFIG);
    int count = 0;
    if (const cudaError_t e = cudaGetDeviceCount(&count)) return cuda_status(e, "cudaGetDeviceCount");
    if (device < 0 || device >= count) return (set_error("device index out of range"), YKB_ERR_INVALID_CONFIG);
    DeviceGuard guard(device);
    int sms = 0;
    YKB_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    DeviceBuffer sink;
    YKB_TRY_CUDA(sink.alloc(sizeof(uint32_t)));
    cudaStream_t s = nullptr;
    YKB_TRY_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    const int blocks = 4 * sms, iters = 4096;
    auto launch = [&]() {
        if (bytes_per_lane == 8)
            shared_load_kernel<2><<<blocks, kProbeThreads, 0, s>>>(iters, sink.as<uint32_t>());
        else
            shared_load_kernel<4><<<blocks, kProbeThreads, 0, s>>>(iters, sink.as<uint32_t>());
        return cudaGetLastError();
    };
    float best = 0.f;
    for (int rep = 0; err == cudaSuccess && rep < 6; ++rep) {
        if ((err = cudaEventRecord(e0, s)) != cudaSuccess || (err = launch()) != cudaSuccess ||
            (err = cudaEventRecord(e1, s)) != cudaSuccess || (err = cudaEventSynchronize(e1)) != cudaSuccess)
            break;
        float ms = 0.f;
        if ((err = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) break;
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;  // the first run warms up
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (err != cudaSuccess) return cuda_status(err, "shared-memory load probe");
    const double bytes = static_cast<double>(blocks) * kProbeThreads * iters * 16.0 * bytes_per_lane;
    *gbs = bytes / (static_cast<double>(best) * 1e-3) / 1e9;
    return YKB_OK;
}
