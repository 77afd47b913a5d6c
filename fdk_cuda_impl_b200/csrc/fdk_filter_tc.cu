// Ramp filter on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// The reference filters each detector row by zero-padded FFT convolution
// (.../FDK/kernels/YkFDKFilterKernels.cu:32-140).  With N >= 2 Nu that is the
// linear product C = A T, A = preweighted rows [rows][Nu], T[k][j] = h(j-k)
// (Toeplitz and, h being even, symmetric).  Here it runs as one BF16 GEMM with
// FP32 accumulation in TMEM and split-precision operands.  Each operand is a
// sum of BF16 parts, X = X0 + X1 (+ X2), each part the BF16 rounding of what
// the previous parts leave; the products are summed over K' = NSEG Nu into
// one accumulator:
//   NSEG 3 (BF16 plans): A0 T0 + A0 T1 + A1 T0, about 16 significant bits;
//   NSEG 6 (FP32 plans): A0 T0 + A0 T1 + A1 T0 + A0 T2 + A1 T1 + A2 T0, the
//     24 bits of FP32 (the dropped products are below 2^-24 of the result).
//     The last three, each at most 2^-18 of |A| |T|, run only over the K
//     chunks near the output tile's columns (`near` chunks each side): the
//     ramp taps fall off as 1/d^2, and the host picks `near` so that the taps
//     beyond carry at most 2^-8 of sum |h|, which leaves what is skipped
//     below the FP32 rounding of the result.
//
// Persistent CTAs, one per SM, walk the output tiles (128 rows x TN
// columns) with six warps:
//   warp 0 lane 0 : TMA producer (A and T tiles, 128-byte swizzle, this
//                   GPU's memory only, no multicast) into a 4-stage ring,
//                   running ahead across tile boundaries;
//   warp 1 lane 0 : MMA issuer (tcgen05.mma kind::f16, M=128, N=TN, K=16)
//                   into one of two TMEM accumulators, releases stages with
//                   tcgen05.commit; warp 1 also owns the TMEM allocation;
//   warps 2-5     : epilogue of the other accumulator, overlapping the next
//                   tile's MMAs: tcgen05.ld of their 32 TMEM lanes, the
//                   placement mask, a transpose through shared memory so that
//                   each global store writes one row's 16 (or 32 tap-pair)
//                   consecutive floats.
// Every mbarrier wait is bounded; on a timeout the CTA records an error,
// drains what it issued, waits for its MMAs to retire and frees its TMEM.
#include "ykb_internal.hpp"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <mutex>

namespace ykb {
namespace {

constexpr int TM = 128, TK = 64, STAGES = 4;
constexpr uint32_t kAStageBytes = TM * TK * 2;  // 16 KiB
constexpr unsigned long long kWaitNs = 2000000000ull;
constexpr int kErrTimeout = 8;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
                 "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(smem_u32(b)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity)
{
    if (bar_try(b, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (!bar_try(b, parity))
        if (now_ns() - t0 > kWaitNs) return false;
    return true;
}
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar)) : "memory");
}

// UMMA shared-memory descriptor of a K-major tile in the 128-byte swizzle
// layout written by TMA: rows of 128 B, 8-row atoms 1024 B apart (SBO),
// descriptor version 1, layout SWIZZLE_128B (2).  The tile base is 1024-byte
// aligned; the k-th 16-element slice starts 32*k bytes further.
__device__ __forceinline__ uint64_t kmajor_sw128_desc(uint32_t saddr)
{
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
        (static_cast<uint64_t>(1024 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
        (static_cast<uint64_t>(2) << 61);
}

// instruction descriptor: D F32, A/B BF16, both K-major, N = TN, M = 128
template <int TN>
__device__ __forceinline__ uint32_t instr_desc()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(TN >> 3) << 17) |
        (static_cast<uint32_t>(TM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
    uint32_t accumulate)
{
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                 " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                 ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate) : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}

// (A part, T part) of segment `seg` of the split product
__device__ __forceinline__ void segment_parts(int seg, int& a, int& t)
{
    // segments 0..5 = (0,0) (0,1) (1,0) (0,2) (1,1) (2,0), one nibble each
    a = (0x210100 >> (4 * seg)) & 0xF;
    t = (0x012010 >> (4 * seg)) & 0xF;
}

// K steps of the output tile starting at column n0: segments 0-2 over all
// kchunks chunks, then (NSEG 6) segments 3-5 over chunks [lo, lo + n)
struct NearChunks { int lo, n; };
template <int TN>
__device__ __forceinline__ NearChunks near_chunks(int n0, int kchunks, int near)
{
    const int c0 = n0 / TK;  // TN is a multiple of TK
    const int lo = max(0, c0 - near), hi = min(kchunks, c0 + TN / TK + near);
    return {lo, max(hi - lo, 0)};
}
template <int NSEG>
__device__ __forceinline__ int tile_steps(int kchunks, NearChunks nc)
{
    return NSEG == 6 ? 3 * kchunks + 3 * nc.n : NSEG * kchunks;
}
__device__ __forceinline__ void step_of(int i, int kchunks, NearChunks nc, int& seg, int& kc)
{
    if (i < 3 * kchunks) {
        seg = i / kchunks;
        kc = i - seg * kchunks;
    } else {
        const int j = i - 3 * kchunks, q = j / nc.n;
        seg = 3 + q;
        kc = nc.lo + j - q * nc.n;
    }
}

static_assert((2 * kPairLead) % 4 == 0, "tap-pair rows start 16-byte aligned after the lead");
constexpr int kEpiWarps = 4;
constexpr int kEpiSplit = kEpiWarps / 4;             // epilogue warps per quarter of the TMEM lanes
constexpr int kFilterThreads = 64 + 32 * kEpiWarps;  // producer, MMA issuer, epilogue warps
constexpr int kStagePitch = 19;                       // floats per staged row: 2 carried + 16 (odd: no bank conflicts)

// 16 consecutive TMEM columns of this warp's 32 lanes, one per register;
// the registers are valid after tmem_wait_ld, which takes them as operands
// so that no use of them is placed before the wait
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[16])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                   "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :: "memory");
}

__device__ __forceinline__ void bar_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

// Persistent CTA (one per SM): tiles t = blockIdx.x + i * gridDim.x of 128
// output rows x TN columns, row tile t / col_tiles, column tile t % col_tiles
// (the column tiles of a row tile run back to back, so its A rows are read
// from L2 while hot).  Two TMEM accumulators: the MMA warp fills one while
// the epilogue warps drain the other.
template <int TN, bool PAIR, int NSEG>
__global__ void __launch_bounds__(kFilterThreads, 1) ramp_tc_kernel(
    const __grid_constant__ CUtensorMap map_a0, const __grid_constant__ CUtensorMap map_a1,
    const __grid_constant__ CUtensorMap map_a2, const __grid_constant__ CUtensorMap map_t0,
    const __grid_constant__ CUtensorMap map_t1, const __grid_constant__ CUtensorMap map_t2,
    long rows, int nu, int nv, int kchunks, int near, int col_tiles, long tiles,
    const FdkPreweightView* __restrict__ pwv, float* __restrict__ C, int ldc, int vec,
    int* __restrict__ err)
{
    constexpr uint32_t kBStageBytes = TN * TK * 2;
    constexpr uint32_t kAccCols = TN <= 32 ? 32 : TN <= 64 ? 64 : TN <= 128 ? 128 : 256;
    constexpr uint32_t kTmemCols = 2 * kAccCols;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char* a_ring = smem;
    unsigned char* b_ring = smem + STAGES * kAStageBytes;
    float* staging = reinterpret_cast<float*>(b_ring + STAGES * kBStageBytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(staging + kEpiWarps * 32 * kStagePitch);
    uint64_t* empty = full + STAGES;
    uint64_t* acc_full = empty + STAGES;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* mma_done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(kTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) { bar_init(&full[s], 1); bar_init(&empty[s], 1); }
        for (int b = 0; b < 2; ++b) { bar_init(&acc_full[b], 1); bar_init(&acc_empty[b], kEpiWarps); }
        bar_init(mma_done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // --------------------------------------------------- producer ---
            long it = 0, issued = 0;
            bool stop = false;
            for (long t = blockIdx.x; t < tiles && !stop; t += gridDim.x) {
                const int m0 = static_cast<int>((t / col_tiles) * TM);
                const int n0 = static_cast<int>((t % col_tiles) * TN);
                const NearChunks nc = near_chunks<TN>(n0, kchunks, near);
                const int total = tile_steps<NSEG>(kchunks, nc);
                for (int i = 0; i < total; ++i, ++it) {
                    const int s = static_cast<int>(it % STAGES);
                    if (it >= STAGES && !bar_wait(&empty[s], static_cast<uint32_t>((it / STAGES) - 1) & 1)) {
                        atomicOr(err, kErrTimeout);
                        *(volatile int*)abort_flag = 1;
                    }
                    if (*(volatile int*)abort_flag) { stop = true; break; }
                    int seg, kc, pa, pt;
                    step_of(i, kchunks, nc, seg, kc);
                    segment_parts(seg, pa, pt);
                    const CUtensorMap* ma = pa == 0 ? &map_a0 : pa == 1 ? &map_a1 : &map_a2;
                    const CUtensorMap* mt = pt == 0 ? &map_t0 : pt == 1 ? &map_t1 : &map_t2;
                    bar_expect_tx(&full[s], kAStageBytes + kBStageBytes);
                    tma_2d(a_ring + s * kAStageBytes, ma, &full[s], kc * TK, m0);
                    tma_2d(b_ring + s * kBStageBytes, mt, &full[s], kc * TK, n0);
                    issued = it + 1;
                }
            }
            // every issued copy must land before the CTA can exit
            for (long j = (issued > STAGES ? issued - STAGES : 0); j < issued; ++j)
                bar_wait(&full[j % STAGES], static_cast<uint32_t>(j / STAGES) & 1);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ------------------------------------------------- MMA issuer ---
            const uint32_t idesc = instr_desc<TN>();
            long it = 0;
            int tl = 0;
            bool stop = false;
            for (long t = blockIdx.x; t < tiles && !stop; t += gridDim.x, ++tl) {
                const int buf = tl & 1;
                // the epilogue has drained this accumulator's previous tile
                if (tl >= 2 && !bar_wait(&acc_empty[buf], static_cast<uint32_t>((tl >> 1) - 1) & 1)) {
                    atomicOr(err, kErrTimeout);
                    *(volatile int*)abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + static_cast<uint32_t>(buf) * kAccCols;
                const int total = tile_steps<NSEG>(kchunks,
                    near_chunks<TN>(static_cast<int>((t % col_tiles) * TN), kchunks, near));
                for (int i = 0; i < total; ++i, ++it) {
                    const int s = static_cast<int>(it % STAGES);
                    if (!bar_wait(&full[s], static_cast<uint32_t>(it / STAGES) & 1)) {
                        atomicOr(err, kErrTimeout);
                        *(volatile int*)abort_flag = 1;
                    }
                    if (*(volatile int*)abort_flag) { stop = true; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint64_t da = kmajor_sw128_desc(smem_u32(a_ring + s * kAStageBytes));
                    const uint64_t db = kmajor_sw128_desc(smem_u32(b_ring + s * kBStageBytes));
#pragma unroll
                    for (int kk = 0; kk < TK / 16; ++kk)
                        mma_bf16(d, da + 2 * kk, db + 2 * kk, idesc, (i > 0 || kk > 0) ? 1u : 0u);
                    mma_commit(&empty[s]);
                }
                if (!stop) mma_commit(&acc_full[buf]);
            }
            // completes when every MMA issued above has retired
            mma_commit(mma_done);
        }
        __syncwarp();
    } else {
        // --------------------------------------------------- epilogue ---
        // warp w reads TMEM lanes 32 (w % 4) ..: rows m0 + 32 (w % 4) + lane,
        // columns [h TW, (h + 1) TW) of the tile, h = (w - 2) / 4.  Eight
        // epilogue warps, or the next chunk's TMEM load issued before this
        // one's stores, measured no faster: both take registers from the
        // preweight that runs beside this kernel
        constexpr int TW = TN / kEpiSplit;
        static_assert(TW % 16 == 0, "whole 16-column chunks per epilogue warp");
        const int q = warp & 3, h = (warp - 2) >> 2;
        float* stg = staging + (warp - 2) * 32 * kStagePitch;
        int tl = 0;
        for (long t = blockIdx.x; t < tiles; t += gridDim.x, ++tl) {
            const int buf = tl & 1;
            // the warp leaves together when a wait runs out
            if (!__all_sync(0xffffffffu, bar_wait(&acc_full[buf], static_cast<uint32_t>(tl >> 1) & 1))) {
                if (lane == 0) {
                    atomicOr(err, kErrTimeout);
                    *(volatile int*)abort_flag = 1;
                }
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const long m0 = (t / col_tiles) * TM;
            const int n0 = static_cast<int>((t % col_tiles) * TN) + h * TW;  // this warp's columns
            const long wrow0 = m0 + q * 32;  // the warp's first row
            const long m = wrow0 + lane;
            // this lane's row keeps columns [lo, hi) (the samples placed in
            // the padded FFT row)
            int lo = 0, hi = 0;
            if (m < rows) {
                const FdkPreweightView& p = pwv[m / nv];
                lo = max(p.out_lo, 0);
                hi = max(min(p.out_hi, nu), lo);
            }
            // tap pairs: this warp writes the floats [X0, X1) of each row
            // (float x holds f[(x + 1) >> 1]): from 2 n0 - 1, or -4 at
            // column 0 (the pairs before the row are zero), up to the next
            // warp's (or tile's) first float, or 2 nu (the right half of the
            // last pair is zero)
            const int X0 = n0 == 0 ? -4 : 2 * n0 - 1;
            const int X1 = n0 + TW >= nu ? 2 * nu : 2 * (n0 + TW) - 1;
            float carry0 = 0.f, carry1 = 0.f;  // columns c0 - 2 and c0 - 1 of the lane's row
            const uint32_t tcol = tmem + (static_cast<uint32_t>(q * 32) << 16) +
                static_cast<uint32_t>(buf) * kAccCols + static_cast<uint32_t>(h * TW);
#pragma unroll 1
            for (int c = 0; c < TW; c += 16) {
                uint32_t r[16];
                tmem_ld16(tcol + static_cast<uint32_t>(c), r);
                tmem_wait_ld(r);
                const int c0 = n0 + c;
                float x[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) x[i] = __uint_as_float(r[i]);
                // the next chunk's load runs while this one is stored

                if (c0 < lo || c0 + 16 > hi) {
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (static_cast<unsigned>(c0 + i - lo) >= static_cast<unsigned>(hi - lo)) x[i] = 0.f;
                }
                // staged row: columns c0 - 2 .. c0 + 15
                float* srow = stg + lane * kStagePitch;
                srow[0] = carry0;
                srow[1] = carry1;
#pragma unroll
                for (int i = 0; i < 16; ++i) srow[2 + i] = x[i];
                carry0 = x[14];
                carry1 = x[15];
                __syncwarp();
                // transposed: each store instruction writes whole row segments
                if constexpr (PAIR) {
                    if (vec) {
                        // 16-byte blocks [xb, xb + 4), xb = 2 c0 - 4 + 4 t:
                        // (f[m], f[m+1], f[m+1], f[m+2]), m = c0 - 2 + 2 t;
                        // eight lanes a row, four rows a store
                        const int t = lane & 7, g = lane >> 3;
                        const int xb = 2 * c0 - 4 + 4 * t;
                        const bool whole = xb >= X0 && xb + 4 <= X1;
                        const bool some = xb + 4 > X0 && xb < X1;
#pragma unroll
                        for (int qq = 0; qq < 8; ++qq) {
                            const int rr = 4 * qq + g;
                            const long mr = wrow0 + rr;
                            if (mr >= rows || !some) continue;
                            const float* sp = stg + rr * kStagePitch + 2 * t;
                            const float a = sp[0], b = sp[1], e = sp[2];
                            float* dst = C + mr * 2 * ldc + 2 * kPairLead + xb;
                            if (whole) {
                                *reinterpret_cast<float4*>(dst) = make_float4(a, b, b, e);
                            } else {
                                if (xb >= X0 && xb < X1) dst[0] = a;
                                if (xb + 1 >= X0 && xb + 1 < X1) dst[1] = b;
                                if (xb + 2 >= X0 && xb + 2 < X1) dst[2] = b;
                                if (xb + 3 >= X0 && xb + 3 < X1) dst[3] = e;
                            }
                        }
                    } else {
                        // lane l writes float 2 c0 - 1 + l, which is f[c0 + l / 2]
                        const int xl = 2 * c0 - 1 + lane;
                        for (int rr = 0; rr < 32; ++rr) {
                            const long mr = wrow0 + rr;
                            if (mr >= rows) break;
                            float* dst = C + mr * 2 * ldc + 2 * kPairLead;
                            if (xl >= X0 && xl < X1) dst[xl] = stg[rr * kStagePitch + 2 + (lane >> 1)];
                            if (c0 == 0 && lane < 3) dst[-4 + lane] = 0.f;
                        }
                    }
                } else {
                    const int xe = min(n0 + TW, nu);  // this warp's columns [n0, xe)
                    if (vec) {
                        // 16-byte blocks: four lanes a row, eight rows a store
                        const int t = lane & 3, g = lane >> 2;
                        const int xb = c0 + 4 * t;
#pragma unroll
                        for (int qq = 0; qq < 4; ++qq) {
                            const int rr = 8 * qq + g;
                            const long mr = wrow0 + rr;
                            if (mr >= rows || xb >= xe) continue;
                            const float* sp = stg + rr * kStagePitch + 2 + 4 * t;
                            float* dst = C + mr * ldc + xb;
                            if (xb + 4 <= xe) {
                                *reinterpret_cast<float4*>(dst) = make_float4(sp[0], sp[1], sp[2], sp[3]);
                            } else {
                                for (int e = 0; e < 4; ++e)
                                    if (xb + e < xe) dst[e] = sp[e];
                            }
                        }
                    } else {
                        const int half = lane >> 4, jj = c0 + (lane & 15);
                        for (int rr = 0; rr < 32; rr += 2) {
                            const long mr = wrow0 + rr + half;
                            if (mr < rows && jj < xe)
                                C[mr * ldc + jj] = stg[(rr + half) * kStagePitch + 2 + (lane & 15)];
                        }
                    }
                }
                __syncwarp();
            }
            if constexpr (PAIR) {
                // the warp's last block, floats 2 (n0 + TW) - 4 .. - 1 =
                // f[n0 + TW - 2], f[n0 + TW - 1] twice, f[n0 + TW]; the last
                // is the next warp's, or zero when the columns end at nu
                if (vec && m < rows) {
                    const int xb = 2 * (n0 + TW) - 4;
                    float* dst = C + m * 2 * ldc + 2 * kPairLead + xb;
                    if (xb >= X0 && xb < X1) dst[0] = carry0;
                    if (xb + 1 >= X0 && xb + 1 < X1) dst[1] = carry1;
                    if (xb + 2 >= X0 && xb + 2 < X1) dst[2] = carry1;
                    if (xb + 3 >= X0 && xb + 3 < X1) dst[3] = 0.f;
                }
            }
            // this accumulator is read out: the MMA warp may refill it
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) bar_arrive(&acc_empty[buf]);
        }
    }
    // teardown: every MMA retired before the TMEM is freed
    __syncwarp();
    if (warp == 1 && lane == 0) bar_wait(mma_done, 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// preweighted rows split into BF16 parts (two, or three when part2 is
// given), rows padded to lda.  One block per row.  The cosine weight is
// D w / |q(iu)| with q(iu) = q0 + iu detU, so |q|^2 = A + iu (B + iu C) with
// the row's A, B, C in FP64 (two FMAs per pixel instead of the vector), then
// an FP32 reciprocal square root refined once in FP64.  A thread takes four
// consecutive pixels: one 16-byte (FP32) or 8-byte (BF16) load when `vec`
// (the input base and row pitch nu keep them aligned), and one 8-byte store
// per part.
struct alignas(8) Bf16x4 { __nv_bfloat16 v[4]; };

__global__ void __launch_bounds__(64) preweight_split_kernel(const void* __restrict__ in,
    int in_bf16, const FdkPreweightView* __restrict__ pw, const float* __restrict__ parker,
    int nu, int nv, int lda, int vec, __nv_bfloat16* __restrict__ part0,
    __nv_bfloat16* __restrict__ part1, __nv_bfloat16* __restrict__ part2)
{
    const long row = blockIdx.x;
    const int view = static_cast<int>(row / nv);
    const int iv = static_cast<int>(row - static_cast<long>(view) * nv);
    const FdkPreweightView& p = pw[view];
    const double qx0 = p.detS[0] + iv * p.detV[0] - p.src[0];
    const double qy0 = p.detS[1] + iv * p.detV[1] - p.src[1];
    const double qz0 = p.detS[2] + iv * p.detV[2] - p.src[2];
    const double A = qx0 * qx0 + qy0 * qy0 + qz0 * qz0;
    const double B = 2.0 * (qx0 * p.detU[0] + qy0 * p.detU[1] + qz0 * p.detU[2]);
    const double Cq = p.detU[0] * p.detU[0] + p.detU[1] * p.detU[1] + p.detU[2] * p.detU[2];
    const double scale = p.dsd * p.wgeom;
    const float* prow = parker ? parker + static_cast<long>(view) * nu : nullptr;
    for (int iu0 = 4 * threadIdx.x; iu0 < lda; iu0 += 4 * blockDim.x) {
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        if (vec && iu0 < nu) {
            if (in_bf16) {
                const uint2 raw = *reinterpret_cast<const uint2*>(
                    static_cast<const __nv_bfloat16*>(in) + row * nu + iu0);
                v[0] = __uint_as_float(raw.x << 16); v[1] = __uint_as_float(raw.x & 0xFFFF0000u);
                v[2] = __uint_as_float(raw.y << 16); v[3] = __uint_as_float(raw.y & 0xFFFF0000u);
            } else {
                const float4 raw = *reinterpret_cast<const float4*>(
                    static_cast<const float*>(in) + row * nu + iu0);
                v[0] = raw.x; v[1] = raw.y; v[2] = raw.z; v[3] = raw.w;
            }
        } else {
            for (int e = 0; e < 4; ++e)
                if (iu0 + e < nu)
                    v[e] = in_bf16
                        ? __bfloat162float(static_cast<const __nv_bfloat16*>(in)[row * nu + iu0 + e])
                        : static_cast<const float*>(in)[row * nu + iu0 + e];
        }
        Bf16x4 h0, h1, h2;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int iu = iu0 + e;
            float x = 0.f;
            if (iu < nu && iu >= p.in_lo && iu < p.in_hi) {
                const double u = static_cast<double>(iu);
                const double r2 = fmax(fma(fma(Cq, u, B), u, A), 1e-20);
                double r = rsqrtf(static_cast<float>(r2));
                r = r * (1.5 - 0.5 * r2 * r * r);
                float wt = static_cast<float>(scale * r);
                if (prow) wt *= prow[iu];
                x = v[e] * wt;
            }
            const __nv_bfloat16 h = __float2bfloat16_rn(x);
            const float r1 = x - __bfloat162float(h);  // exact
            const __nv_bfloat16 m = __float2bfloat16_rn(r1);
            h0.v[e] = h;
            h1.v[e] = m;
            h2.v[e] = __float2bfloat16_rn(r1 - __bfloat162float(m));
        }
        *reinterpret_cast<Bf16x4*>(part0 + row * lda + iu0) = h0;
        *reinterpret_cast<Bf16x4*>(part1 + row * lda + iu0) = h1;
        if (part2) *reinterpret_cast<Bf16x4*>(part2 + row * lda + iu0) = h2;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 tma_encode()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

bool make_map(CUtensorMap* map, const void* base, long inner, long outer, long ld_elems, int box_inner,
    int box_outer)
{
    auto enc = tma_encode();
    if (!enc) return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(inner), static_cast<cuuint64_t>(outer)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld_elems) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_inner), static_cast<cuuint32_t>(box_outer)};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int TN, bool PAIR, int NSEG>
cudaError_t launch_tn3(const CUtensorMap* a, const CUtensorMap* t, long rows, int nu, int nv,
    int kchunks, int near, const FdkPreweightView* pwv, float* C, int ldc, int* err, cudaStream_t s)
{
    // 16-byte stores need the rows 16-byte aligned: tap-pair rows are
    // 2 ldc floats with kPairLead pairs before element 0
    const int vec = reinterpret_cast<uintptr_t>(C) % 16 == 0 && ldc % (PAIR ? 2 : 4) == 0;
    const size_t smem = 1024 + STAGES * (kAStageBytes + TN * TK * 2) +
        kEpiWarps * 32 * kStagePitch * sizeof(float) + (2 * STAGES + 5) * 8 + 16;
    auto k = ramp_tc_kernel<TN, PAIR, NSEG>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
        static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0;
    if ((e = cudaGetDevice(&device)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return e;
    const int col_tiles = (nu + TN - 1) / TN;
    const long tiles = static_cast<long>(col_tiles) * ((rows + TM - 1) / TM);
    const unsigned grid = static_cast<unsigned>(std::min<long>(tiles, sms));
    k<<<grid, kFilterThreads, smem, s>>>(a[0], a[1], a[2], t[0], t[1], t[2], rows, nu, nv,
        kchunks, near, col_tiles, tiles, pwv, C, ldc, vec, err);
    return cudaGetLastError();
}

template <int TN, bool PAIR>
cudaError_t launch_tn(const CUtensorMap* a, const CUtensorMap* t, int nseg, long rows, int nu,
    int nv, int kchunks, int near, const FdkPreweightView* pwv, float* C, int ldc, int* err,
    cudaStream_t s)
{
    return nseg == 6 ? launch_tn3<TN, PAIR, 6>(a, t, rows, nu, nv, kchunks, near, pwv, C, ldc, err, s)
                     : launch_tn3<TN, PAIR, 3>(a, t, rows, nu, nv, kchunks, near, pwv, C, ldc, err, s);
}

} // namespace

int tc_filter_tile_n(int nu)
{
    // fewest padded columns, then the widest tile
    int best = 0;
    long best_cols = 0;
    for (int tn : {256, 192, 128, 64}) {
        const long cols = static_cast<long>((nu + tn - 1) / tn) * tn;
        if (best == 0 || cols < best_cols) { best = tn; best_cols = cols; }
    }
    return best;
}

bool tcgen05_filter_supported(int nu) { return tma_encode() != nullptr && nu >= 16; }

int tc_filter_lda(int nu) { return (nu + TK - 1) / TK * TK; }

int tc_filter_near_chunks(const std::vector<double>& h, int nu)
{
    // h[nu - 1 + d] = h(d), d in (-nu, nu); a tile skips, in its 2^-16
    // products, only lags |d| > near * TK
    const int kchunks = (nu + TK - 1) / TK;
    double total = 0.0;
    for (double v : h) total += std::fabs(v);
    for (int near = 1; near < kchunks; ++near) {
        double tail = 0.0;
        for (int d = near * TK + 1; d < nu; ++d)
            tail += std::fabs(h[static_cast<size_t>(nu - 1 + d)]) +
                std::fabs(h[static_cast<size_t>(nu - 1 - d)]);
        if (tail <= total / 256.0) return near;
    }
    return kchunks;
}

cudaError_t launch_fdk_preweight_split_bf16(const void* proj, int proj_dtype,
    const FdkPreweightView* pw, const float* parker, int n_views, int nu, int nv, int ld,
    __nv_bfloat16* const parts[3], cudaStream_t s)
{
    const long rows = static_cast<long>(n_views) * nv;
    if (rows <= 0) return cudaSuccess;
    if (ld % 4 != 0) return cudaErrorInvalidValue;  // rows are padded to whole K chunks
    const bool bf16 = proj_dtype == YKB_DTYPE_BF16;
    const int vec = nu % 4 == 0 && reinterpret_cast<uintptr_t>(proj) % (bf16 ? 8 : 16) == 0;
    preweight_split_kernel<<<static_cast<unsigned>(rows), 64, 0, s>>>(proj, bf16 ? 1 : 0, pw,
        parker, nu, nv, ld, vec, parts[0], parts[1], parts[2]);
    return cudaGetLastError();
}

cudaError_t launch_fdk_ramp_tcgen05(const __nv_bfloat16* const a_parts[3],
    const __nv_bfloat16* const t_parts[3], int rows, int nu, int ld, const FdkPreweightView* pwv,
    int nv, float* out, int layout, int ldc, int near_chunks, int* err, cudaStream_t s)
{
    if (rows <= 0) return cudaSuccess;
    const int tn = tc_filter_tile_n(nu);
    const int nparts = a_parts[2] && t_parts[2] ? 3 : 2;
    CUtensorMap a[3], t[3];
    // A: [rows][ld] K-major, box 64 x 128; T: [nu][ld] K-major, box 64 x TN
    for (int q = 0; q < 3; ++q) {
        const int src = q < nparts ? q : 0;  // an unused slot repeats part 0
        if (!make_map(&a[q], a_parts[src], nu, rows, ld, TK, TM) ||
            !make_map(&t[q], t_parts[src], nu, nu, ld, TK, tn))
            return cudaErrorInvalidValue;
    }
    const int nseg = nparts == 3 ? 6 : 3;
    const int kchunks = (nu + TK - 1) / TK;
    const int near = std::min(std::max(near_chunks, 1), kchunks);
    const bool pair = layout == kFilteredPairs;
    switch (tn) {
    case 256: return pair ? launch_tn<256, true>(a, t, nseg, rows, nu, nv, kchunks, near, pwv, out, ldc, err, s)
                          : launch_tn<256, false>(a, t, nseg, rows, nu, nv, kchunks, near, pwv, out, ldc, err, s);
    case 192: return pair ? launch_tn<192, true>(a, t, nseg, rows, nu, nv, kchunks, near, pwv, out, ldc, err, s)
                          : launch_tn<192, false>(a, t, nseg, rows, nu, nv, kchunks, near, pwv, out, ldc, err, s);
    case 128: return pair ? launch_tn<128, true>(a, t, nseg, rows, nu, nv, kchunks, near, pwv, out, ldc, err, s)
                          : launch_tn<128, false>(a, t, nseg, rows, nu, nv, kchunks, near, pwv, out, ldc, err, s);
    default: return pair ? launch_tn<64, true>(a, t, nseg, rows, nu, nv, kchunks, near, pwv, out, ldc, err, s)
                         : launch_tn<64, false>(a, t, nseg, rows, nu, nv, kchunks, near, pwv, out, ldc, err, s);
    }
}

} // namespace ykb
