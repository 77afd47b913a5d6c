// FDK weighted backprojection with TMA-staged projection tiles (sm_100a).
//
// Same arithmetic as fdk_bp_kernel in fdk_kernels.cu (the math of
// .../FDK/kernels/YkFDKBpKernels.cu:112-209 with exact software bilinear
// weights), organised for Blackwell:
//   * a CTA owns a 16x32x64 voxel tile, one CTA per SM; each of its 512
//     consumer threads walks a 64-voxel z-column and keeps the 64 sums in
//     registers over all views (the longer the column, the more voxels share
//     the per-view column terms); a remainder of at most 32 slices runs as
//     32-voxel columns, the same launch's last z layer.  Against two CTAs of
//     16x16x48 per SM: the same warps per SM, a third more voxels per
//     column, and one ring of ~200 KB whose stages each feed twice the
//     columns, so the copies run further ahead of the consumers (62.2 ->
//     60.4 ms on the 512^3 x 720 x 768^2 workload);
//   * one producer warp computes, per view, the detector box covering the
//     tile's footprint (+1 bilinear tap, +1 pixel margin) and loads it with
//     cp.async.bulk.tensor (3D tile mode, this GPU's memory only, no
//     multicast) into a ring of shared-memory stages guarded by full/empty
//     mbarriers.  Out-of-detector box elements are zero-filled by TMA, which
//     is the reference's Border addressing;
//   * filtered rows arrive either as plain floats or as tap pairs, element
//     (v, kPairLead + u) = (f[v][u], f[v][u+1]), zero outside the detector
//     (written so by the filter epilogues).  With pairs one 8-byte shared
//     load returns both horizontal taps of a detector row, and the vertical
//     lerp runs as one packed f32x2 operation on the (left, right) pair;
//   * consumers read the four taps from shared memory without bounds checks:
//     the box is sized by a pre-pass over all (tile, view) pairs with the same
//     footprint function, and each (column, view) checks its end points.
// Every mbarrier wait is bounded (~2 s of %globaltimer by default; the
// pipeline waits take the limit as a kernel argument, so that a test can
// shorten it); a timeout sets the plan's error word, stops the CTA and drains
// the copies in flight, each drain wait with the full limit.
#include "ykb_internal.hpp"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

namespace ykb {
namespace {

constexpr int TX = 16, TY = 32, ZT = 64;
constexpr int kZTail = 32;  // column length of a short last z tile
constexpr int NCONS = TX * TY;          // consumer threads
constexpr int NCWARPS = NCONS / 32;
constexpr int NTHREADS = NCONS + 32;    // + producer warp
constexpr unsigned long long kWaitNs = 2000000000ull;

// error word bits
constexpr int kErrTimeout = 1;
constexpr int kErrFootprint = 2;
constexpr int kErrAlign = 4;

// a TMA tile copy writes shared memory at 128-byte aligned addresses: each
// stage starts on a 128-byte boundary
__host__ __device__ constexpr int stage_stride_floats(int bw, int bh, bool pair)
{
    return (bw * bh * (pair ? 2 : 1) + 31) / 32 * 32;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// bounded wait: false after limit_ns
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
    unsigned long long limit_ns = kWaitNs)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
    int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ double rcp64(double x)
{
    double r = static_cast<double>(__frcp_rn(static_cast<float>(x)));
    return r * (2.0 - x * r);
}

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two z-voxels per instruction.
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
template <int OFF>
__device__ __forceinline__ float lds(uint32_t addr)
{
    float v;
    asm("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(addr), "n"(OFF));
    return v;
}
// one tap pair (8-byte aligned)
template <int OFF>
__device__ __forceinline__ f2 lds2(uint32_t addr)
{
    f2 v;
    asm("ld.shared.b64 %0, [%1+%2];" : "=l"(v) : "r"(addr), "n"(OFF));
    return v;
}

// floor by rounding: t = (v - 1/2) + 1.5*2^23 holds round(v - 1/2) in its
// low mantissa bits for |v| < 2^22, and round(v - 1/2) = floor(v) except at
// integer v, where it may give v - 1 with fraction 1 -- the same bilinear
// value.  The map v -> t is monotonic.
constexpr float kRoundMagic = 12582912.0f;
constexpr uint32_t kRoundMagicBits = 0x4B400000u;

// Per (column, view) terms of the axial path, independent of the staged box:
// computed one view ahead so their FP64 latency overlaps the previous view.
// PSEUDO (pseudo-matched weight ks L(i) / den^2): w = ks / den^2 and
// L(i)^2 = alp + i (bet + i gam) along the column, the detector quadratic
// L^2(u, v) of PseudoViewCoef evaluated at u and v(i) = vb + i vs.
struct ColTerms {
    float u, vbq, vs, w;
    float alp, bet, gam;
};

template <bool PSEUDO>
__device__ __forceinline__ ColTerms axial_terms(const FdkViewCoef& c, const PseudoViewCoef* pc,
    double X, double Y, double Z0, double vz)
{
    const double den = fma(c.cd[1], Y, fma(c.cd[0], X, c.cd[3]));
    const double rd = rcp64(den);
    const double un = fma(c.cu[1], Y, fma(c.cu[0], X, c.cu[3]));
    const double vn = fma(c.cv[2], Z0, fma(c.cv[1], Y, fma(c.cv[0], X, c.cv[3])));
    ColTerms t;
    const double u = un * rd, vb = vn * rd, vs = c.cv[2] * vz * rd;
    t.u = static_cast<float>(u);
    t.vbq = static_cast<float>(vb - 0.5);
    t.vs = static_cast<float>(vs);
    if constexpr (PSEUDO) {
        const float* l = pc->l2;
        const double A = fma(u, fma(u, static_cast<double>(l[3]), static_cast<double>(l[1])),
                             static_cast<double>(l[0]));
        const double B = fma(u, static_cast<double>(l[4]), static_cast<double>(l[2]));
        const double C = l[5];
        t.alp = static_cast<float>(fma(vb, fma(vb, C, B), A));
        t.bet = static_cast<float>(fma(2.0 * C, vb, B) * vs);
        t.gam = static_cast<float>(C * vs * vs);
        t.w = static_cast<float>(static_cast<double>(pc->ks) * rd * rd);
    } else {
        const double dep = fma(c.cr[1], Y, fma(c.cr[0], X, c.cr[3]));
        const double rdep = rcp64(dep);
        t.w = static_cast<float>(c.wbase * rdep * rdep);
        t.alp = t.bet = t.gam = 0.f;
    }
    return t;
}

__device__ __forceinline__ float sqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Detector box of a voxel tile for one view: columns [c0, c1], rows [r0, r1]
// covering every bilinear tap of the tile's voxel centres with two pixels of
// margin each side, c0 rounded down to the TMA alignment (16 bytes).  The
// pre-pass and the producer evaluate the same corners with the same code.
struct Box { int c0, c1, r0, r1; };

__device__ __forceinline__ void corner_uv(const FdkViewCoef& c, double X, double Y, double Z,
    double& u, double& v)
{
    const double den = fma(c.cd[2], Z, fma(c.cd[1], Y, fma(c.cd[0], X, c.cd[3])));
    const double r = rcp64(den);
    u = fma(c.cu[2], Z, fma(c.cu[1], Y, fma(c.cu[0], X, c.cu[3]))) * r;
    v = fma(c.cv[2], Z, fma(c.cv[1], Y, fma(c.cv[0], X, c.cv[3]))) * r;
}

__device__ __forceinline__ Box box_from_range(double umin, double umax, double vmin, double vmax)
{
    umin = fmax(umin, -1e8); umax = fmin(umax, 1e8);
    vmin = fmax(vmin, -1e8); vmax = fmin(vmax, 1e8);
    Box b;
    b.c0 = (static_cast<int>(floor(umin)) - 2) & ~3;
    b.c1 = static_cast<int>(floor(umax)) + 3;
    b.r0 = static_cast<int>(floor(vmin)) - 2;
    b.r1 = static_cast<int>(floor(vmax)) + 3;
    return b;
}

struct TileGeom {
    double x0, x1, y0, y1, z0, z1;
    double xc, yc;  // centre of the nominal TX x TY tile (reference point of its column terms)
};

__device__ __forceinline__ TileGeom tile_geom(const VolumeGrid& g, int bx, int by, int za, int zc)
{
    TileGeom t;
    const int xa = bx * TX, ya = by * TY;
    t.x0 = g.ox + xa * g.vx;
    t.x1 = g.ox + min(xa + TX - 1, g.nx - 1) * g.vx;
    t.y0 = g.oy + ya * g.vy;
    t.y1 = g.oy + min(ya + TY - 1, g.ny - 1) * g.vy;
    t.z0 = g.oz + za * g.vz;
    t.z1 = g.oz + (za + zc - 1) * g.vz;  // all zc slices are evaluated
    t.xc = g.ox + (xa + 0.5 * (TX - 1)) * g.vx;
    t.yc = g.oy + (ya + 0.5 * (TY - 1)) * g.vy;
    return t;
}

// Pre-pass: largest box over all (tile, view) pairs.
__global__ void box_extent_kernel(const FdkViewCoef* __restrict__ coef, int n_views, VolumeGrid g,
    int tiles_x, int tiles_y, int tiles_z, int* __restrict__ out)
{
    const long n = static_cast<long>(tiles_x) * tiles_y * tiles_z * n_views;
    int w = 0, h = 0;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const int k = static_cast<int>(i % n_views);
        const long t = i / n_views;
        const int bx = static_cast<int>(t % tiles_x);
        const int by = static_cast<int>((t / tiles_x) % tiles_y);
        const int bz = static_cast<int>(t / (static_cast<long>(tiles_x) * tiles_y));
        const TileGeom tg = tile_geom(g, bx, by, bz * ZT, ZT);
        double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
        for (int q = 0; q < 8; ++q) {
            double u, v;
            corner_uv(coef[k], (q & 1) ? tg.x1 : tg.x0, (q & 2) ? tg.y1 : tg.y0,
                (q & 4) ? tg.z1 : tg.z0, u, v);
            umin = fmin(umin, u); umax = fmax(umax, u);
            vmin = fmin(vmin, v); vmax = fmax(vmax, v);
        }
        const Box b = box_from_range(umin, umax, vmin, vmax);
        w = max(w, b.c1 - b.c0 + 1);
        h = max(h, b.r1 - b.r0 + 1);
    }
    atomicMax(out, w);
    atomicMax(out + 1, h);
}

// Per-(tile, view) terms of the FDK axial path, FP64-derived by the producer
// and stored beside the view's stage; each consumer evaluates its column's
// terms from them in FP32.  With d = (X - xc, Y - yc) the column's offset
// from the tile centre and P = (X, Y, z0) its first voxel:
//   den = dc + gd . d                      (cd . P)
//   u   = uc + (hu . d) / den              hu = (cu_x, cu_y) - u_c (cd_x, cd_y)
//   vq  = vc + (hv . d) / den              hv = (cv_x, cv_y) - v_c (cd_x, cd_y)
//   vs  = kz / den                         kz = cv_z vz, one slice up
//   w   = wbase / dep^2,  dep = pc + gp . d (cr . P)
// exact rewrites of u = cu.P / cd.P and v = cv.P / cd.P about the tile
// centre (the numerators of u - u_c and v - v_c vanish there).  u and vq are
// relative to the staged box (pixel c0; row r0, minus the 1/2 of the row
// rounding), so they stay below the box size and round to within 4e-6 px.
struct alignas(16) TileTerms {
    float uc, hu0, hu1, vc;
    float hv0, hv1, dc, gd0;
    float gd1, kz, pc, gp0;
    float gp1, wbase, unused0, unused1;
};

__device__ __forceinline__ TileTerms tile_terms(const FdkViewCoef& c, const TileGeom& tg,
    double vz, int c0, int r0)
{
    const double den = fma(c.cd[1], tg.yc, fma(c.cd[0], tg.xc, c.cd[3]));
    const double rd = 1.0 / den;
    const double uc = fma(c.cu[1], tg.yc, fma(c.cu[0], tg.xc, c.cu[3])) * rd;
    const double vc = fma(c.cv[2], tg.z0, fma(c.cv[1], tg.yc, fma(c.cv[0], tg.xc, c.cv[3]))) * rd;
    const double dep = fma(c.cr[1], tg.yc, fma(c.cr[0], tg.xc, c.cr[3]));
    TileTerms t;
    t.uc = static_cast<float>(uc - c0);
    t.hu0 = static_cast<float>(c.cu[0] - uc * c.cd[0]);
    t.hu1 = static_cast<float>(c.cu[1] - uc * c.cd[1]);
    t.vc = static_cast<float>(vc - r0 - 0.5);
    t.hv0 = static_cast<float>(c.cv[0] - vc * c.cd[0]);
    t.hv1 = static_cast<float>(c.cv[1] - vc * c.cd[1]);
    t.dc = static_cast<float>(den);
    t.gd0 = static_cast<float>(c.cd[0]);
    t.gd1 = static_cast<float>(c.cd[1]);
    t.kz = static_cast<float>(c.cv[2] * vz);
    t.pc = static_cast<float>(dep);
    t.gp0 = static_cast<float>(c.cr[0]);
    t.gp1 = static_cast<float>(c.cr[1]);
    t.wbase = static_cast<float>(c.wbase);
    t.unused0 = t.unused1 = 0.f;
    return t;
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Shared-memory ring budget of the one CTA of an SM.
constexpr size_t kRingBudget = 200 * 1024;

// Shared memory of the backprojection CTA: the ring of stages, their
// full/empty barriers, and per stage the staged box and (FDK axial tap-pair
// path) the producer's tile terms of its view.
struct BpSmem {
    float* ring;
    uint64_t* full;
    uint64_t* empty;
    int4* boxes;
    TileTerms* terms;
    int* abort_flag;
    int stage_floats;
};

__device__ __forceinline__ BpSmem bp_smem(int BW, int BH, bool pair, int stages)
{
    extern __shared__ unsigned char smem_raw[];
    // 128-byte aligned base (the launch requests 128 bytes of slack)
    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
    BpSmem m;
    m.stage_floats = stage_stride_floats(BW, BH, pair);
    const size_t ring_bytes = static_cast<size_t>(m.stage_floats) * sizeof(float) * stages;
    m.ring = reinterpret_cast<float*>(smem);
    m.full = reinterpret_cast<uint64_t*>(smem + ring_bytes);
    m.empty = m.full + stages;
    m.boxes = reinterpret_cast<int4*>(m.empty + stages);
    m.terms = reinterpret_cast<TileTerms*>(m.boxes + stages);
    m.abort_flag = reinterpret_cast<int*>(m.terms + stages);
    return m;
}

// Tiles in order: layers of TX x TY tiles (x fastest), the ZT-slice layers
// from slice 0, then at most one layer of kZTail-slice tiles (a short last
// part of the volume; it lies inside the ZT-slice layer of the box pre-pass,
// so its footprints fit the same box).
struct TileId { int bx, by, za; bool main; };

__device__ __forceinline__ TileId tile_id(long t, int tiles_x, int tiles_y, int main_tiles)
{
    const long per_layer = static_cast<long>(tiles_x) * tiles_y;
    const int bz = static_cast<int>(t / per_layer);
    const int rem = static_cast<int>(t - bz * per_layer);
    TileId id;
    id.by = rem / tiles_x;
    id.bx = rem - id.by * tiles_x;
    id.main = bz < main_tiles;
    id.za = id.main ? bz * ZT : main_tiles * ZT + (bz - main_tiles) * kZTail;
    return id;
}

// The consumer warps' part of one tile (bx, by, slices from za).  The stage
// index s and its phase run on across the CTA's tiles.  False when a wait
// ran out (the CTA stops).
// PSEUDO: the weight of the pseudo-matched backprojection instead of the FDK
// depth weight (tap pairs only)
template <int BW, bool AXIAL, bool PAIR, bool PSEUDO, int ZC, bool ACC>
__device__ __forceinline__ bool bp_consume(const BpSmem& sm,
    const FdkViewCoef* __restrict__ coef, int n_views, const VolumeGrid& g, int BH, int stages,
    float* __restrict__ vol, int* __restrict__ err,
    const PseudoViewCoef* __restrict__ pseudo, int bx, int by, int za, PipelineWait pw, int& s,
    uint32_t& phase)
{
    constexpr bool COLS = AXIAL && PAIR && !PSEUDO;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    // --------------------------------------------------------- consumers ---
    // a warp covers an 8x4 block of columns, each half-warp a 4x4 block: the
    // detector footprint of 16 lanes then spans few columns, so the 16-lane
    // phases of 8-byte shared loads (and 32-lane 4-byte ones) rarely share
    // a bank
    const int lx = 8 * (warp & 1) + 4 * (lane >> 4) + (lane & 3);
    const int ly = 4 * (warp >> 1) + ((lane >> 2) & 3);
    const int x = bx * TX + lx, y = by * TY + ly;
    const int z0 = za;
    const bool active = x < g.nx && y < g.ny;
    const double X = g.ox + x * g.vx, Y = g.oy + y * g.vy, Z0 = g.oz + z0 * g.vz;
    float acc[ZC];
#pragma unroll
    for (int i = 0; i < ZC; ++i) acc[i] = 0.f;
    bool bad = false;
    ColTerms cur{};
    if (AXIAL && !COLS) cur = axial_terms<PSEUDO>(coef[0], pseudo, X, Y, Z0, g.vz);
    // the column's offset from the tile centre (exact: a few voxel pitches)
    float dx = 0.f, dy = 0.f;
    if constexpr (COLS) {
        const TileGeom tg = tile_geom(g, bx, by, za, ZC);
        dx = static_cast<float>(X - tg.xc);
        dy = static_cast<float>(Y - tg.yc);
    }

    for (int k = 0; k < n_views; ++k, (++s == stages ? (s = 0, phase ^= 1u) : 0)) {
        // the warp leaves together: a lane whose wait ran out takes its whole
        // warp with it, so no lane is left waiting at the warp barrier below
        if (!__all_sync(0xffffffffu, mbar_wait(&sm.full[s], phase, pw.limit_ns))) {
            if (lane == 0) {
                atomicOr(err, kErrTimeout);
                *(volatile int*)sm.abort_flag = 1;
            }
            return false;
        }
        const float* S = sm.ring + static_cast<size_t>(s) * sm.stage_floats;
        if constexpr (COLS) {
            // the column's terms in FP32 from the tile terms of this view
            const TileTerms& T = sm.terms[s];
            const float4 t0 = *reinterpret_cast<const float4*>(&T.uc);
            const float4 t1 = *reinterpret_cast<const float4*>(&T.hv0);
            const float4 t2 = *reinterpret_cast<const float4*>(&T.gd1);
            const float2 t3 = *reinterpret_cast<const float2*>(&T.gp1);
            const float den = fmaf(t2.x, dy, fmaf(t1.w, dx, t1.z));
            float rd = rcp_approx(den);
            rd = fmaf(rd, fmaf(-den, rd, 1.f), rd);  // one Newton step: vs walks 64 slices
            float u = fmaf(fmaf(t0.z, dy, t0.y * dx), rd, t0.x);
            float vbq = fmaf(fmaf(t1.y, dy, t1.x * dx), rd, t0.w);
            float vs = t2.y * rd;
            const float dep = fmaf(t3.x, dy, fmaf(t2.w, dx, t2.z));
            const float rp = rcp_approx(dep);
            float w = t3.y * rp * rp;
            const float fu = floorf(u);
            int col = static_cast<int>(fu);
            float au = u - fu;
            // rows of the column's end points (the rounding map is monotonic)
            const int na = static_cast<int>(__float_as_uint(vbq + kRoundMagic) - kRoundMagicBits);
            const int nb = static_cast<int>(__float_as_uint(fmaf(static_cast<float>(ZC - 1), vs, vbq) +
                kRoundMagic) - kRoundMagicBits);
            // every tap inside the staged BW x BH box (it holds the detector's
            // values, zero outside the detector); |v| < 2^21 keeps the
            // rounding word exact
            const bool inside = fabsf(u) < 1e6f && fabsf(vbq) < 1e6f && fabsf(vs) < 3e4f &&
                w < 1e30f && col >= 0 && col <= BW - 1 && min(na, nb) >= 0 && max(na, nb) <= BH - 2;
            if (!active || !inside) {
                if (active) bad = true;
                // no contribution; every read stays at the stage origin
                w = 0.f; au = 0.f; vs = 0.f; vbq = 0.f;
                col = 0;
            }
            const uint32_t base = smem_addr(S) + 8u * static_cast<uint32_t>(col) -
                8u * BW * kRoundMagicBits;
            const float w1 = w * au, w0 = w - w1;
            const f2 M2 = f2pack(kRoundMagic, kRoundMagic), H2 = f2pack(0.5f, 0.5f);
#pragma unroll
            for (int j = 0; j < ZC / 2; ++j) {
                const f2 vq = f2pack(fmaf(2.f * j, vs, vbq), fmaf(2.f * j + 1.f, vs, vbq));
                const f2 t = f2add(vq, M2);
                const f2 fr = f2add(f2sub(vq, f2sub(t, M2)), H2);
                float t0f, t1f, f0, f1;
                f2unpack(t, t0f, t1f);
                f2unpack(fr, f0, f1);
                const uint32_t a0 = __float_as_uint(t0f) * (8u * BW) + base;
                const uint32_t a1 = __float_as_uint(t1f) * (8u * BW) + base;
                const f2 A0 = lds2<0>(a0), B0 = lds2<8 * BW>(a0);
                const f2 A1 = lds2<0>(a1), B1 = lds2<8 * BW>(a1);
                // vertical lerps as scalar FMAs on the halves of the pairs
                // (a packed FMA would need each fraction in both halves)
                float al0, ar0, dl0, dr0, al1, ar1, dl1, dr1;
                f2unpack(A0, al0, ar0);
                f2unpack(f2sub(B0, A0), dl0, dr0);
                f2unpack(A1, al1, ar1);
                f2unpack(f2sub(B1, A1), dl1, dr1);
                const float l0 = fmaf(f0, dl0, al0), r0 = fmaf(f0, dr0, ar0);
                const float l1 = fmaf(f1, dl1, al1), r1 = fmaf(f1, dr1, ar1);
                acc[2 * j] = fmaf(w1, r0, fmaf(w0, l0, acc[2 * j]));
                acc[2 * j + 1] = fmaf(w1, r1, fmaf(w0, l1, acc[2 * j + 1]));
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.empty[s]);
            continue;
        }
        const int4 b = sm.boxes[s];
        const FdkViewCoef& c = coef[k];
        if (AXIAL) {
            // next view's terms first: independent of this view's stage
            const ColTerms nxt = (k + 1 < n_views)
                ? axial_terms<PSEUDO>(coef[k + 1], pseudo + (PSEUDO ? k + 1 : 0), X, Y, Z0, g.vz)
                : cur;
            const float u = cur.u;
            const float fu = floorf(u);
            const int iu = static_cast<int>(fu);
            float au = u - fu;
            float vbq = cur.vbq, vs = cur.vs, w = cur.w;
            float alp = cur.alp, bet = cur.bet, gam = cur.gam;
            // rows of the column's end points (the rounding map is monotonic)
            const int na = static_cast<int>(__float_as_uint(vbq + kRoundMagic) - kRoundMagicBits);
            const int nb = static_cast<int>(__float_as_uint(fmaf(static_cast<float>(ZC - 1), vs, vbq) +
                kRoundMagic) - kRoundMagicBits);
            const int lo = min(na, nb), hi = max(na, nb) + 1;
            // |v| < 2^21 along the column keeps the rounding word exact
            const bool finite = fabsf(u) < 1e6f && fabsf(vbq) < 1e6f && fabsf(vs) < 3e4f &&
                fabsf(w) < 1e30f && (!PSEUDO || (alp > 0.f && alp < 1e30f &&
                fmaf(static_cast<float>(ZC - 1), fmaf(static_cast<float>(ZC - 1), gam, bet), alp) > 0.f &&
                fabsf(bet) < 1e30f && fabsf(gam) < 1e30f));
            int col = iu - b.x;
            if (!active || !finite || iu < b.x || iu + 1 > b.z || lo < b.y || hi > b.w) {
                if (active) bad = true;
                // no contribution; every read stays at the stage origin
                w = 0.f; au = 0.f; vs = 0.f;
                alp = 1.f; bet = 0.f; gam = 0.f;
                vbq = static_cast<float>(b.y);
                col = 0;
            }
            // smem byte address of tap (row n, col) = n*4BW + base, n taken
            // from the rounding word (wrapping 32-bit arithmetic)
            constexpr uint32_t ES = PAIR ? 8u : 4u;  // bytes per staged element
            const uint32_t base = smem_addr(S) + ES * static_cast<uint32_t>(col) -
                ES * BW * (static_cast<uint32_t>(b.y) + kRoundMagicBits);
            // the column's horizontal weights, with the view weight folded in
            const float w1 = w * au, w0 = w - w1;
            const f2 M2 = f2pack(kRoundMagic, kRoundMagic), H2 = f2pack(0.5f, 0.5f);
            if constexpr (PSEUDO) {
                // L(i) is a square root of a quadratic in i; the FP64 column
                // terms keep its sqrt argument positive along the column
#pragma unroll
                for (int j = 0; j < ZC / 2; ++j) {
                    const float i0 = 2.f * j, i1 = 2.f * j + 1.f;
                    const f2 vq = f2pack(fmaf(i0, vs, vbq), fmaf(i1, vs, vbq));
                    const f2 t = f2add(vq, M2);
                    const f2 fr = f2add(f2sub(vq, f2sub(t, M2)), H2);
                    float t0, t1, f0, f1;
                    f2unpack(t, t0, t1);
                    f2unpack(fr, f0, f1);
                    const uint32_t a0 = __float_as_uint(t0) * (8u * BW) + base;
                    const uint32_t a1 = __float_as_uint(t1) * (8u * BW) + base;
                    const f2 A0 = lds2<0>(a0), B0 = lds2<8 * BW>(a0);
                    const f2 A1 = lds2<0>(a1), B1 = lds2<8 * BW>(a1);
                    float l0, r0, l1, r1;
                    f2unpack(f2fma(f2pack(f0, f0), f2sub(B0, A0), A0), l0, r0);
                    f2unpack(f2fma(f2pack(f1, f1), f2sub(B1, A1), A1), l1, r1);
                    const float L0 = sqrt_approx(fmaf(i0, fmaf(i0, gam, bet), alp));
                    const float L1 = sqrt_approx(fmaf(i1, fmaf(i1, gam, bet), alp));
                    acc[2 * j] = fmaf(w * L0, fmaf(au, r0 - l0, l0), acc[2 * j]);
                    acc[2 * j + 1] = fmaf(w * L1, fmaf(au, r1 - l1, l1), acc[2 * j + 1]);
                }
            } else if constexpr (PAIR) {
#pragma unroll
                for (int j = 0; j < ZC / 2; ++j) {
                    const f2 vq = f2pack(fmaf(2.f * j, vs, vbq), fmaf(2.f * j + 1.f, vs, vbq));
                    const f2 t = f2add(vq, M2);
                    const f2 fr = f2add(f2sub(vq, f2sub(t, M2)), H2);
                    float t0, t1, f0, f1;
                    f2unpack(t, t0, t1);
                    f2unpack(fr, f0, f1);
                    const uint32_t a0 = __float_as_uint(t0) * (8u * BW) + base;
                    const uint32_t a1 = __float_as_uint(t1) * (8u * BW) + base;
                    // rows n and n+1, each (left, right): lerp down as a pair,
                    // then weight across into the voxel's sum
                    const f2 A0 = lds2<0>(a0), B0 = lds2<8 * BW>(a0);
                    const f2 A1 = lds2<0>(a1), B1 = lds2<8 * BW>(a1);
                    float l0, r0, l1, r1;
                    f2unpack(f2fma(f2pack(f0, f0), f2sub(B0, A0), A0), l0, r0);
                    f2unpack(f2fma(f2pack(f1, f1), f2sub(B1, A1), A1), l1, r1);
                    acc[2 * j] = fmaf(w1, r0, fmaf(w0, l0, acc[2 * j]));
                    acc[2 * j + 1] = fmaf(w1, r1, fmaf(w0, l1, acc[2 * j + 1]));
                }
            } else {
#pragma unroll
            for (int j = 0; j < ZC / 2; ++j) {
                // rows and vertical weights of z = 2j, 2j+1 in packed pairs;
                // the taps themselves stay scalar so that no load result has
                // to be moved into a register pair
                const f2 vq = f2pack(fmaf(2.f * j, vs, vbq), fmaf(2.f * j + 1.f, vs, vbq));
                const f2 t = f2add(vq, M2);
                const f2 d = f2sub(vq, f2sub(t, M2));  // in [-1/2, 1/2]
                const f2 fr = f2add(d, H2), gr = f2sub(H2, d);
                float t0, t1, f0, f1, g0, g1;
                f2unpack(t, t0, t1);
                f2unpack(fr, f0, f1);
                f2unpack(gr, g0, g1);
                const uint32_t a0 = __float_as_uint(t0) * (4u * BW) + base;
                const uint32_t a1 = __float_as_uint(t1) * (4u * BW) + base;
                const float h00 = fmaf(w1, lds<4>(a0), w0 * lds<0>(a0));
                const float h01 = fmaf(w1, lds<4 * BW + 4>(a0), w0 * lds<4 * BW>(a0));
                const float h10 = fmaf(w1, lds<4>(a1), w0 * lds<0>(a1));
                const float h11 = fmaf(w1, lds<4 * BW + 4>(a1), w0 * lds<4 * BW>(a1));
                acc[2 * j] = fmaf(f0, h01, fmaf(g0, h00, acc[2 * j]));
                acc[2 * j + 1] = fmaf(f1, h11, fmaf(g1, h10, acc[2 * j + 1]));
            }
            }
            cur = nxt;
        } else {
            const double den0 = fma(c.cd[2], Z0, fma(c.cd[1], Y, fma(c.cd[0], X, c.cd[3])));
            const double un0 = fma(c.cu[2], Z0, fma(c.cu[1], Y, fma(c.cu[0], X, c.cu[3])));
            const double vn0 = fma(c.cv[2], Z0, fma(c.cv[1], Y, fma(c.cv[0], X, c.cv[3])));
            const double dp0 = fma(c.cr[2], Z0, fma(c.cr[1], Y, fma(c.cr[0], X, c.cr[3])));
            const float s0 = PSEUDO ? 1.f : static_cast<float>(c.wbase);
            const float dn = static_cast<float>(den0), ddn = static_cast<float>(c.cd[2] * g.vz);
            const float uu = static_cast<float>(un0), dun = static_cast<float>(c.cu[2] * g.vz);
            const float vv = static_cast<float>(vn0), dvn = static_cast<float>(c.cv[2] * g.vz);
            const float dp = static_cast<float>(dp0), ddp = static_cast<float>(c.cr[2] * g.vz);
            // end points: u(z) and v(z) are monotonic along the column
            const float ra = 1.f / dn, rb = 1.f / fmaf(ZC - 1.f, ddn, dn);
            const float ua = uu * ra, ub = fmaf(ZC - 1.f, dun, uu) * rb;
            const float va = vv * ra, vb2 = fmaf(ZC - 1.f, dvn, vv) * rb;
            // u(z), v(z) are monotonic; one row/column of slack covers the
            // rounding of the interior samples
            const int ulo = static_cast<int>(floorf(fminf(ua, ub))) - 1;
            const int uhi = static_cast<int>(floorf(fmaxf(ua, ub))) + 2;
            const int vlo = static_cast<int>(floorf(fminf(va, vb2))) - 1;
            const int vhi = static_cast<int>(floorf(fmaxf(va, vb2))) + 2;
            float scale = s0;
            float gdn = dn, gddn = ddn, guu = uu, gdun = dun, gvv = vv, gdvn = dvn, gdp = dp, gddp = ddp;
            const bool finite = fabsf(ua) < 1e7f && fabsf(ub) < 1e7f && fabsf(va) < 1e7f &&
                fabsf(vb2) < 1e7f && dn > 0.f && fmaf(ZC - 1.f, ddn, dn) > 0.f &&
                dp > 0.f && fmaf(ZC - 1.f, ddp, dp) > 0.f;
            if (!active || !finite || ulo < b.x || uhi > b.z || vlo < b.y || vhi > b.w) {
                if (active) bad = true;
                scale = 0.f;  // no contribution; reads stay at the stage origin
                gdn = 1.f; gddn = 0.f; guu = static_cast<float>(b.x); gdun = 0.f;
                gvv = static_cast<float>(b.y); gdvn = 0.f; gdp = 1.f; gddp = 0.f;
            }
            const int cb = -b.x - b.y * BW;
#pragma unroll
            for (int i = 0; i < ZC; ++i) {
                const float fi = static_cast<float>(i);
                const float rden = 1.f / fmaf(fi, gddn, gdn);
                const float u = fmaf(fi, gdun, guu) * rden;
                const float v = fmaf(fi, gdvn, gvv) * rden;
                float w;
                if constexpr (PSEUDO) {
                    // ks L / den^2 (the reference's k L^3 / |P - S|^2 on the ray)
                    const PseudoViewCoef& pv = pseudo[k];
                    const float L2 = fmaf(v, fmaf(v, pv.l2[5], fmaf(u, pv.l2[4], pv.l2[2])),
                                          fmaf(u, fmaf(u, pv.l2[3], pv.l2[1]), pv.l2[0]));
                    w = L2 > 1e-8f ? scale * pv.ks * sqrt_approx(L2) * rden * rden : 0.f;
                } else {
                    const float rdep = 1.f / fmaf(fi, gddp, gdp);
                    w = scale * rdep * rdep;
                }
                const float fu = floorf(u), fv = floorf(v);
                const int a = static_cast<int>(fv) * BW + static_cast<int>(fu) + cb;
                const float au = u - fu, av = v - fv;
                float p00, p10, p01, p11;
                if constexpr (PAIR) {
                    const float2* S2 = reinterpret_cast<const float2*>(S);
                    const float2 A = S2[a], B = S2[a + BW];
                    p00 = A.x; p10 = A.y; p01 = B.x; p11 = B.y;
                } else {
                    p00 = S[a]; p10 = S[a + 1]; p01 = S[a + BW]; p11 = S[a + BW + 1];
                }
                const float r0 = fmaf(au, p10 - p00, p00);
                const float r1 = fmaf(au, p11 - p01, p01);
                acc[i] = fmaf(w, fmaf(av, r1 - r0, r0), acc[i]);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.empty[s]);
    }
    if (bad) atomicOr(err, kErrFootprint);
    if (!active) return true;
    const long plane = static_cast<long>(g.nx) * g.ny;
    float* dst = vol + static_cast<long>(y) * g.nx + x;
    if constexpr (ACC) {
        // a reduction in L2 (each voxel has this one writer, so the sum is the
        // plain old + acc): no load round trip per value, which one after
        // another cost about 1 ms per 512^3 launch
#pragma unroll
        for (int i = 0; i < ZC; ++i) {
            const int z = z0 + i;
            if (z < g.nz) atomicAdd(dst + z * plane, acc[i]);
        }
    } else {
#pragma unroll
        for (int i = 0; i < ZC; ++i) {
            const int z = z0 + i;
            if (z < g.nz) dst[z * plane] = acc[i];
        }
    }
    return true;
}

// Persistent: one CTA of 17 warps per SM walks tiles blockIdx.x, +gridDim.x,
// ... (see tile_id).  The producer warp runs on into the next tile's views
// while the consumers finish a tile and write its sums, so a tile costs no
// pipeline fill or drain of its own (a CTA per tile cost about 0.8 ms per
// 512^3 launch in starting and ending 4096 CTAs).  Registers are granted for
// whole groups of four warps (20 here), which caps a thread at 96: enough
// for the 64 sums of the axial tap-pair path (a few bytes of spill); the
// other paths spill more.
// ACC: add to the volume instead of writing it (a separate kernel, so that
// the write-only form's registers are not shaped by the reductions)
template <int BW, bool AXIAL, bool PAIR, bool PSEUDO, bool ACC>
__global__ void __launch_bounds__(NTHREADS, 1) fdk_bp_tma_kernel(const __grid_constant__ CUtensorMap map,
    const FdkViewCoef* __restrict__ coef, int n_views, VolumeGrid g, int BH, int stages,
    float* __restrict__ vol, int* __restrict__ err,
    const PseudoViewCoef* __restrict__ pseudo, int main_tiles, int tiles_x, int tiles_y,
    long n_tiles, PipelineWait pw)
{
    constexpr bool COLS = AXIAL && PAIR && !PSEUDO;
    const BpSmem sm = bp_smem(BW, BH, PAIR, stages);
    const uint32_t box_bytes = static_cast<uint32_t>(BW * BH * (PAIR ? 8 : 4));
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        *sm.abort_flag = 0;
        if ((smem_addr(sm.full) & 7u) != 0 || (smem_addr(sm.ring) & 127u) != 0) {
            atomicOr(err, kErrAlign);
            *sm.abort_flag = 1;
        }
        for (int s = 0; s < stages; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], NCWARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (*sm.abort_flag) return;

    if (warp == NCWARPS) {
        // ------------------------------------------------------ producer ---
        // lanes 0..7 project one tile corner each; lane 0 owns the barriers.
        // q counts the CTA's copies over all its tiles: stage q % stages,
        // used q / stages times before
        long q = 0, issued = 0;
        bool ok = true;
        for (long t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
            const TileId id = tile_id(t, tiles_x, tiles_y, main_tiles);
            const TileGeom tg = tile_geom(g, id.bx, id.by, id.za, id.main ? ZT : kZTail);
            for (int k = 0; k < n_views; ++k, ++q) {
                const int s = static_cast<int>(q % stages);
                const long use = q / stages;
                // the view's box and terms first, while the consumers still
                // read the stage: only the copy waits for it to be released
                double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
                if (lane < 8) {
                    corner_uv(coef[k], (lane & 1) ? tg.x1 : tg.x0, (lane & 2) ? tg.y1 : tg.y0,
                        (lane & 4) ? tg.z1 : tg.z0, umin, vmin);
                    umax = umin; vmax = vmin;
                }
#pragma unroll
                for (int o = 4; o > 0; o >>= 1) {
                    umin = fmin(umin, __shfl_xor_sync(0xffffffffu, umin, o));
                    umax = fmax(umax, __shfl_xor_sync(0xffffffffu, umax, o));
                    vmin = fmin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
                    vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
                }
                const Box b = box_from_range(umin, umax, vmin, vmax);
                TileTerms tt{};
                if constexpr (COLS)
                    if (lane == 0) tt = tile_terms(coef[k], tg, g.vz, b.c0, b.r0);
                int go = 1;
                if (lane == 0) {
                    if (use > 0 && !mbar_wait(&sm.empty[s], static_cast<uint32_t>(use - 1) & 1u,
                            pw.limit_ns))
                        go = 0;
                    if (*(volatile int*)sm.abort_flag) go = 0;
                }
                go = __shfl_sync(0xffffffffu, go, 0);
                if (!go) { ok = false; break; }
                if (k == pw.withheld_view) {
                    // test hook: no copy and no arrival for this view, so every
                    // wait for it runs out
                    issued = q + 1;
                    continue;
                }
                int aligned = 1;
                if (lane == 0) {
                    float* dst = sm.ring + static_cast<size_t>(s) * sm.stage_floats;
                    if ((smem_addr(dst) & 127u) != 0 || (b.c0 & 3) != 0) {
                        aligned = 0;  // never issue a copy the hardware would reject
                    } else {
                        sm.boxes[s] = make_int4(b.c0, b.r0, b.c1, b.r1);
                        if constexpr (COLS) sm.terms[s] = tt;
                        mbar_arrive_expect_tx(&sm.full[s], box_bytes);
                        tma_load_3d(dst, &map, &sm.full[s], b.c0 + (PAIR ? kPairLead : 0), b.r0, k);
                    }
                }
                aligned = __shfl_sync(0xffffffffu, aligned, 0);
                if (!aligned) {
                    if (lane == 0) atomicOr(err, kErrAlign);
                    ok = false;
                    break;
                }
                issued = q + 1;
            }
        }
        if (!ok && lane == 0) {
            atomicOr(err, kErrTimeout);
            *(volatile int*)sm.abort_flag = 1;
            // drain: every issued copy must land before the CTA exits
            for (long j = max(0L, issued - stages); j < issued; ++j)
                if (static_cast<int>(j % n_views) != pw.withheld_view)
                    mbar_wait(&sm.full[j % stages], static_cast<uint32_t>(j / stages) & 1u);
        }
        return;
    }

    // --------------------------------------------------------- consumers ---
    int s = 0;
    uint32_t phase = 0;
    for (long t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const TileId id = tile_id(t, tiles_x, tiles_y, main_tiles);
        const bool ok = id.main
            ? bp_consume<BW, AXIAL, PAIR, PSEUDO, ZT, ACC>(sm, coef, n_views, g, BH, stages, vol,
                  err, pseudo, id.bx, id.by, id.za, pw, s, phase)
            : bp_consume<BW, AXIAL, PAIR, PSEUDO, kZTail, ACC>(sm, coef, n_views, g, BH, stages,
                  vol, err, pseudo, id.bx, id.by, id.za, pw, s, phase);
        if (!ok) return;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
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

// Staged box widths (elements).  Each is 8 mod 16, so a row of tap pairs is
// 64 mod 128 bytes: the 16 lanes of a half-warp, whose footprints span a few
// columns and at most a row or two, then rarely meet on one bank (a pitch of
// 32 mod 128 bytes put rows n and n + 1 four pairs apart on the same banks:
// 16 % more shared-memory wavefronts, measured).
constexpr int kWidths[] = {40, 56, 72, 104, 136, 200, 248};
// Widths 4 narrower, for the axial tap-pair FDK kernel only: taken when the
// narrower stage leaves room for one more ring stage (a third stage beats
// the better bank pattern: 1081 vs 1491 ms on the 1024^3 x 1440 workload,
// whose 52-wide box needs 3 stages of 34.5 KB).  The other kernels launch
// such a box at the next width of kWidths.
constexpr int kNarrowWidths[] = {36, 52, 68, 100, 132, 196};

// z tiling: ZT-slice tiles, except that a remainder of at most kZTail
// slices becomes one kZTail-slice tile instead of a ZT-slice tile that is
// mostly outside the volume (see tile_id).
template <typename K>
cudaError_t launch_kernel(K k, const CUtensorMap& map, const FdkViewCoef* coef, int n_views,
    const VolumeGrid& g, int BH, int stages, size_t smem, float* vol, int accumulate, int* err,
    const PseudoViewCoef* pseudo, PipelineWait pw, cudaStream_t s)
{
    const int rem = g.nz % ZT;
    const bool tail = rem > 0 && rem <= kZTail;
    const int main_tiles = tail ? g.nz / ZT : (g.nz + ZT - 1) / ZT;
    const int tiles_x = (g.nx + TX - 1) / TX, tiles_y = (g.ny + TY - 1) / TY;
    const long n_tiles = static_cast<long>(tiles_x) * tiles_y * (main_tiles + (tail ? 1 : 0));
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
        static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0;
    if ((e = cudaGetDevice(&device)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return e;
    // one persistent CTA per SM (the ring takes most of its shared memory)
    const unsigned grid = static_cast<unsigned>(std::min<long>(n_tiles, sms));
    k<<<grid, NTHREADS, smem, s>>>(map, coef, n_views, g, BH, stages, vol, err, pseudo,
        main_tiles, tiles_x, tiles_y, n_tiles, pw);
    return cudaGetLastError();
}

template <int BW, bool PAIR>
cudaError_t launch_bw(const CUtensorMap& map, const FdkViewCoef* coef, int n_views,
    const VolumeGrid& g, int BH, int stages, size_t smem, bool axial, float* vol, int accumulate,
    int* err, const PseudoViewCoef* pseudo, PipelineWait pw, cudaStream_t s)
{
    if constexpr (PAIR) {
        if (pseudo && axial)
            return launch_kernel(accumulate ? fdk_bp_tma_kernel<BW, true, true, true, true> : fdk_bp_tma_kernel<BW, true, true, true, false>, map, coef, n_views, g,
                BH, stages, smem, vol, accumulate, err, pseudo, pw, s);
        if (pseudo)
            return launch_kernel(accumulate ? fdk_bp_tma_kernel<BW, false, true, true, true> : fdk_bp_tma_kernel<BW, false, true, true, false>, map, coef, n_views, g,
                BH, stages, smem, vol, accumulate, err, pseudo, pw, s);
    } else {
        if (pseudo) return cudaErrorInvalidValue;  // pseudo-matched input is staged as pairs
    }
    if (axial)
        return launch_kernel(accumulate ? fdk_bp_tma_kernel<BW, true, PAIR, false, true> : fdk_bp_tma_kernel<BW, true, PAIR, false, false>, map, coef, n_views, g, BH,
            stages, smem, vol, accumulate, err, pseudo, pw, s);
    return launch_kernel(accumulate ? fdk_bp_tma_kernel<BW, false, PAIR, false, true> : fdk_bp_tma_kernel<BW, false, PAIR, false, false>, map, coef, n_views, g, BH,
        stages, smem, vol, accumulate, err, pseudo, pw, s);
}

template <int BW>
cudaError_t launch_narrow(const CUtensorMap& map, const FdkViewCoef* coef, int n_views,
    const VolumeGrid& g, int BH, int stages, size_t smem, float* vol, int accumulate, int* err,
    PipelineWait pw, cudaStream_t s)
{
    return launch_kernel(accumulate ? fdk_bp_tma_kernel<BW, true, true, false, true> : fdk_bp_tma_kernel<BW, true, true, false, false>, map, coef, n_views, g, BH,
        stages, smem, vol, accumulate, err, nullptr, pw, s);
}

template <bool PAIR>
cudaError_t launch_layout(const CUtensorMap& map, const FdkViewCoef* coef, int n_views,
    const VolumeGrid& g, int bw, int bh, int stages, size_t smem, bool axial, float* vol,
    int accumulate, int* err, const PseudoViewCoef* pseudo, PipelineWait pw, cudaStream_t s)
{
    switch (bw) {
    case 40: return launch_bw<40, PAIR>(map, coef, n_views, g, bh, stages, smem, axial, vol, accumulate, err, pseudo, pw, s);
    case 56: return launch_bw<56, PAIR>(map, coef, n_views, g, bh, stages, smem, axial, vol, accumulate, err, pseudo, pw, s);
    case 72: return launch_bw<72, PAIR>(map, coef, n_views, g, bh, stages, smem, axial, vol, accumulate, err, pseudo, pw, s);
    case 104: return launch_bw<104, PAIR>(map, coef, n_views, g, bh, stages, smem, axial, vol, accumulate, err, pseudo, pw, s);
    case 136: return launch_bw<136, PAIR>(map, coef, n_views, g, bh, stages, smem, axial, vol, accumulate, err, pseudo, pw, s);
    case 200: return launch_bw<200, PAIR>(map, coef, n_views, g, bh, stages, smem, axial, vol, accumulate, err, pseudo, pw, s);
    case 248: return launch_bw<248, PAIR>(map, coef, n_views, g, bh, stages, smem, axial, vol, accumulate, err, pseudo, pw, s);
    default: break;
    }
    if constexpr (PAIR) {
        if (axial && !pseudo) {
            switch (bw) {
            case 36: return launch_narrow<36>(map, coef, n_views, g, bh, stages, smem, vol, accumulate, err, pw, s);
            case 52: return launch_narrow<52>(map, coef, n_views, g, bh, stages, smem, vol, accumulate, err, pw, s);
            case 68: return launch_narrow<68>(map, coef, n_views, g, bh, stages, smem, vol, accumulate, err, pw, s);
            case 100: return launch_narrow<100>(map, coef, n_views, g, bh, stages, smem, vol, accumulate, err, pw, s);
            case 132: return launch_narrow<132>(map, coef, n_views, g, bh, stages, smem, vol, accumulate, err, pw, s);
            case 196: return launch_narrow<196>(map, coef, n_views, g, bh, stages, smem, vol, accumulate, err, pw, s);
            default: break;
            }
        }
    }
    return cudaErrorInvalidValue;
}

} // namespace

// Largest tile box over all views and tiles; returns the chosen width (one of
// kWidths or kNarrowWidths, 0 if none fits) and height.
cudaError_t fdk_tma_box(const FdkViewCoef* coef, int n_views, const VolumeGrid& g, int* scratch2,
    int* bw, int* bh, cudaStream_t s)
{
    *bw = 0; *bh = 0;
    cudaError_t e = cudaMemsetAsync(scratch2, 0, 2 * sizeof(int), s);
    if (e != cudaSuccess) return e;
    const int tx = (g.nx + TX - 1) / TX, ty = (g.ny + TY - 1) / TY, tz = (g.nz + ZT - 1) / ZT;
    box_extent_kernel<<<1184, 256, 0, s>>>(coef, n_views, g, tx, ty, tz, scratch2);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int host[2] = {0, 0};
    if ((e = cudaMemcpyAsync(host, scratch2, sizeof host, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    *bh = host[1];
    if (*bh > 256) return cudaSuccess;
    for (int w : kWidths)
        if (w >= host[0]) { *bw = w; break; }
    // the narrower width when it fits the box and buys a ring stage while the
    // wider one still runs (2 stages or more) for the other kernels
    const int wide = fdk_tma_stages(*bw, *bh, kFilteredPairs);
    for (int w : kNarrowWidths)
        if (w == *bw - 4 && w >= host[0] && wide >= 2 &&
            fdk_tma_stages(w, *bh, kFilteredPairs) > wide)
            *bw = w;
    return cudaSuccess;
}

int fdk_tma_z_tile() { return ZT; }

// Stages that fit the shared-memory budget for a box (0 when fewer than 2).
int fdk_tma_stages(int bw, int bh, int layout)
{
    const size_t stage = static_cast<size_t>(
        stage_stride_floats(bw, bh, layout == kFilteredPairs)) * sizeof(float);
    int s = static_cast<int>(kRingBudget / std::max<size_t>(stage, 1));
    s = std::min(s, 8);
    return s >= 2 ? s : 0;
}

bool fdk_tma_available() { return encode_fn() != nullptr; }

cudaError_t launch_fdk_backproject_tma(const float* filtered, int layout, int ld,
    int rows_total_views, const FdkViewCoef* coef, int n_views, int nu, int nv,
    const VolumeGrid& g, bool axial, int bw, int bh, float* vol, int accumulate, int* err,
    cudaStream_t s, const PseudoViewCoef* pseudo, PipelineWait pw)
{
    auto enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const bool pair = layout == kFilteredPairs;
    if (bw % 16 == 4 && !(pair && axial && !pseudo)) bw += 4;  // a narrow width: see kNarrowWidths
    const size_t esz = pair ? 8 : 4;  // a tap pair moves as one 8-byte element
    CUtensorMap map;
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(pair ? nu + kPairLead : nu),
                                static_cast<cuuint64_t>(nv),
                                static_cast<cuuint64_t>(rows_total_views)};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(ld) * esz,
                                   static_cast<cuuint64_t>(ld) * nv * esz};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(bw), static_cast<cuuint32_t>(bh), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(&map,
        pair ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
        const_cast<float*>(filtered), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const int stages = fdk_tma_stages(bw, bh, layout);
    if (stages == 0) return cudaErrorInvalidConfiguration;
    const size_t ring = static_cast<size_t>(stage_stride_floats(bw, bh, pair)) * sizeof(float) * stages;
    const size_t smem = 128 + ring + 2 * stages * sizeof(uint64_t) +
        stages * (sizeof(int4) + sizeof(TileTerms)) + 16;
    return pair ? launch_layout<true>(map, coef, n_views, g, bw, bh, stages, smem, axial, vol,
                      accumulate, err, pseudo, pw, s)
                : launch_layout<false>(map, coef, n_views, g, bw, bh, stages, smem, axial, vol,
                      accumulate, err, pseudo, pw, s);
}

// Scalar filtered rows [rows][ld_in] -> tap pairs [rows][ldp]: element
// kPairLead + u = (f[u], f[u+1]) for u in [-kPairLead, nu), zero outside the
// row -- the layout the filter epilogues write directly.
__global__ void pairify_kernel(const float* __restrict__ in, int ld_in, long rows, int nu,
    float2* __restrict__ out, int ldp)
{
    const int width = nu + kPairLead;
    const long n = rows * width;
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long>(gridDim.x) * blockDim.x) {
        const long r = i / width;
        const int u = static_cast<int>(i - r * width) - kPairLead;
        const float* row = in + r * ld_in;
        out[r * ldp + u + kPairLead] = make_float2(u >= 0 ? row[u] : 0.f,
            u + 1 >= 0 && u + 1 < nu ? row[u + 1] : 0.f);
    }
}

cudaError_t launch_fdk_pairify(const float* in, int ld_in, long rows, int nu, float* out,
    int ldp, cudaStream_t s)
{
    if (rows <= 0) return cudaSuccess;
    pairify_kernel<<<148 * 8, 256, 0, s>>>(in, ld_in, rows, nu, reinterpret_cast<float2*>(out), ldp);
    return cudaGetLastError();
}

} // namespace ykb
