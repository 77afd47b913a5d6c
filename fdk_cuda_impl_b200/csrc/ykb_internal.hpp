// Internal declarations shared by the host and CUDA translation units of
// libykb.so.  Nothing here crosses the C-ABI.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "ykb.h"

namespace ykb {

// --------------------------------------------------------------- errors ---
void set_error(const std::string& msg);
void clear_error();
const char* last_error();

// Returns YKB_ERR_CUDA (and records the message) when status is an error.
ykb_status cuda_status(cudaError_t status, const char* what);

#define YKB_TRY_CUDA(expr)                                                   \
    do {                                                                     \
        const cudaError_t ykb_e_ = (expr);                                   \
        if (ykb_e_ != cudaSuccess) return ::ykb::cuda_status(ykb_e_, #expr); \
    } while (0)

// Device buffer owned by a plan (RAII; no exceptions).
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { reset(); }
    cudaError_t alloc(size_t n)
    {
        reset();
        if (n == 0) return cudaSuccess;
        const cudaError_t e = cudaMalloc(&ptr, n);
        if (e == cudaSuccess) bytes = n; else ptr = nullptr;
        return e;
    }
    void reset()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// Switches to a device for the lifetime of the object and restores the
// caller's device afterwards.
struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device)
    {
        if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
        if (previous != device) cudaSetDevice(device);
    }
    ~DeviceGuard()
    {
        int now = -1;
        if (previous >= 0 && cudaGetDevice(&now) == cudaSuccess && now != previous)
            cudaSetDevice(previous);
    }
};

// ------------------------------------------------------------- geometry ---
struct dvec3 { double x, y, z; };

// Per-view FDK quantities derived in FP64 from the float geometry
// (definitions of src/Reconstruction/Analytic/Circular/Flat/FDK/
// YkFDKVecGeoDerived.hpp:58-304).
struct FdkDerived {
    double theta, dtheta, fscale;
    double sid;     // source_to_axis_mm
    double dsd;     // source_to_radial_detector_mm
    double plane;   // source_to_detector_plane_mm
    double off_u, off_v;
    double du, dv;
    dvec3 src, detS, detU, detV, normal, radial;
    double UU, VV, UV, inv_gram;
    int start_u;    // placement of the row inside the padded FFT row
};

bool derive_fdk_geometry(const ykb_cone_view* views, int n, int nu, int nv,
    float scan_range, std::vector<FdkDerived>& out, std::string& why);

int padded_fft_length(int nu);

// Device-side per-view FDK coefficients (FP64).  Affine rows over world
// coordinates (X, Y, Z, 1): u = cu.P/cd.P, v = cv.P/cd.P (pixel units,
// pixel (0,0) at detS), radial depth = cr.P; wbase = SID^2 dtheta 2pi/range.
struct alignas(16) FdkViewCoef {
    double cu[4];
    double cv[4];
    double cd[4];
    double cr[4];
    double wbase;
    double pad[3];
};

// Device-side per-view preweight + placement data.
struct alignas(16) FdkPreweightView {
    double src[4];
    double detS[4];
    double detU[4];
    double detV[4];
    double dsd;     // cosine-weight numerator
    double wgeom;   // DSD / DSO / 2
    int in_lo, in_hi;   // input samples [in_lo, in_hi) are placed in the padded row
    int out_lo, out_hi; // outputs [out_lo, out_hi) fall inside the padded row
};

bool build_parker_weights(const std::vector<FdkDerived>& g, const ykb_cone_view* views, int nu,
    int nv, double scan_range, double start_angle, int direction, std::vector<float>& w,
    std::string& why);
void build_fdk_coefficients(const std::vector<FdkDerived>& g, int nu,
    std::vector<FdkViewCoef>& coef, std::vector<FdkPreweightView>& pw,
    bool& axial);

void build_ramp_kernel(int nu, double du, const ykb_filter& f,
    std::vector<double>& h);

// Per-view data of the pseudo-matched backprojection (BP_FDK_PseudoMatched,
// src/FlatFpBp/BP/kernels/YkBpFdkKernel.cu:356-450).  A voxel P projecting to
// detector pixel coordinates (u, v) receives k L^3 / |P - S|^2 times the
// bilinear sample, where L^2 = |detS + u detU + v detV - S|^2 is expanded
// once per view as a quadratic in (u, v) and k = voxel volume /
// (du dv |SDD_plane|) (src/Reconstruction/Analytic/Circular/Flat/FDK/kernels/
// YkFDKBpPrecompute.cu:104-122).
// Since |P - S| = L den / SDD_plane for the detector point of P (den =
// (P - S).n, n the unit detector normal), the weight equals
// ks L / den^2 with ks = voxel volume |SDD_plane| / (du dv); the TMA
// kernel uses that form, in which only L varies along an axial z-column.
struct alignas(16) PseudoViewCoef {
    double src[4];
    float l2[6];  // l2[0] + u l2[1] + v l2[2] + u^2 l2[3] + u v l2[4] + v^2 l2[5]
    float k;
    float ks;
};

void build_pseudo_coefficients(const std::vector<FdkDerived>& g, const ykb_volume& vol,
    std::vector<PseudoViewCoef>& out);

// Joseph per-view data (FP64), volume-centred voxel units.
struct alignas(16) JosephView {
    double src[4];
    double detS[4];
    double detU[4];
    double detV[4];
    int axis;        // 0: X main axis, 1: Y, 2: Z
    int n0, n1, n2;  // volume extents along (main, minor1, minor2)
    double v0, v1, v2;  // voxel sizes (mm) along the same axes
    double pad;
};

bool build_joseph_views(const ykb_cone_view* views, int n, int nu, int nv,
    const ykb_volume& vol, std::vector<JosephView>& out, std::string& why);

bool build_circular_flat(const ykb_circular_flat& spec, ykb_cone_view* out,
    std::string& why);

// -------------------------------------------------------------- kernels ---
struct VolumeGrid {
    int nx, ny, nz;
    double vx, vy, vz;
    double ox, oy, oz;  // centre of voxel (0,0,0), FP64
};

VolumeGrid make_grid(const ykb_volume& v);

// FDK
// Layouts of filtered rows: plain floats [row][ld], or tap pairs
// [row][ld] float2 where element kPairLead + u = (f[u], f[u+1]) for
// u in [-kPairLead, nu) with f outside [0, nu) = 0.  The TMA
// backprojection reads a row's two horizontal taps with one 8-byte load;
// the two leading pairs keep the TMA box origin 16-byte aligned while
// u = -1 still sees (0, f[0]).
enum FilteredLayout : int { kFilteredScalar = 0, kFilteredPairs = 1 };
constexpr int kPairLead = 2;
// parker: per-(view, column) weights [n_views][nu] multiplied in after the
// cosine weight (short scans), or nullptr
cudaError_t launch_fdk_preweight(const void* proj, int proj_dtype,
    const FdkPreweightView* pw, const float* parker, int n_views, int nu, int nv, float* out,
    cudaStream_t s);
cudaError_t launch_fdk_ramp_fp32(const float* pw_rows, const float* h_dev,
    const FdkPreweightView* pwv, int n_views, int nu, int nv, float* out,
    int layout, int ldc, cudaStream_t s);
// BF16 split parts of the preweighted rows: parts[0], parts[1] and, when
// parts[2] is not null, a third part (FP32-equivalent split)
cudaError_t launch_fdk_preweight_split_bf16(const void* proj, int proj_dtype,
    const FdkPreweightView* pw, const float* parker, int n_views, int nu, int nv, int ld,
    __nv_bfloat16* const parts[3], cudaStream_t s);
// tcgen05 Toeplitz filter over split operands: two parts each (3 products,
// BF16 plans) or three (6 products, FP32 accuracy) when a_parts[2] and
// t_parts[2] are given.  With three parts the three products at the 2^-16
// level run only over the K chunks (64 columns each) within `near_chunks`
// chunks of each output tile; tc_filter_near_chunks(h, nu) picks the
// fewest chunks for which the filter taps left out carry at most 2^-8 of
// the taps' absolute sum.
cudaError_t launch_fdk_ramp_tcgen05(const __nv_bfloat16* const a_parts[3],
    const __nv_bfloat16* const t_parts[3], int rows, int nu, int ld,
    const FdkPreweightView* pwv, int nv, float* out, int layout, int ldc, int near_chunks,
    int* err_flag, cudaStream_t s);
int tc_filter_near_chunks(const std::vector<double>& h, int nu);
bool tcgen05_filter_supported(int nu);
int tc_filter_lda(int nu);
cudaError_t launch_fdk_backproject(const void* filtered, int dtype,
    const FdkViewCoef* coef, int n_views, int nu, int nv, int ld,
    const VolumeGrid& grid, bool axial, float* vol, int accumulate,
    cudaStream_t s);
// TMA-staged backprojection (fdk_bp_tma.cu)
bool fdk_tma_available();
int fdk_tma_stages(int bw, int bh, int layout);
// z slices per tile of the TMA backprojection (slab work starts on a tile)
int fdk_tma_z_tile();
cudaError_t fdk_tma_box(const FdkViewCoef* coef, int n_views, const VolumeGrid& g,
    int* scratch2, int* bw, int* bh, cudaStream_t s);
// Limit of the TMA backprojection's pipeline waits (a wait that runs out
// sets the error word and stops the CTA) and, for tests of that path, a view
// whose copy the producer withholds (-1: none).  Waits that drain copies in
// flight keep the default limit.
struct PipelineWait {
    unsigned long long limit_ns = 2000000000ull;
    int withheld_view = -1;
};
// pseudo != nullptr: the pseudo-matched weight of PseudoViewCoef replaces the
// FDK depth weight (tap-pair layout only)
cudaError_t launch_fdk_backproject_tma(const float* filtered, int layout, int ld,
    int views_in_buffer, const FdkViewCoef* coef, int n_views, int nu, int nv,
    const VolumeGrid& g, bool axial, int bw, int bh, float* vol, int accumulate, int* err,
    cudaStream_t s, const PseudoViewCoef* pseudo = nullptr, PipelineWait pw = PipelineWait{});
// Pseudo-matched backprojection straight from projections [n][nv][nu] with
// bounds-checked loads (used when the TMA box does not fit)
cudaError_t launch_pseudo_backproject(const float* proj, const FdkViewCoef* coef,
    const PseudoViewCoef* pseudo, int n_views, int nu, int nv, const VolumeGrid& grid,
    float* vol, int accumulate, cudaStream_t s);
cudaError_t launch_fdk_pairify(const float* in, int ld_in, long rows, int nu, float* out,
    int ldp, cudaStream_t s);

// Joseph
// zero voxels bordering each slice of the transposed slabs on both minor axes
constexpr int kSlabPad = 2;
// slab of main axis x ([x][z][y]) or y ([y][z][x]) with its zero border
inline size_t joseph_slab_elems(const ykb_volume& v, int axis)
{
    const size_t n0 = static_cast<size_t>(axis == 0 ? v.nx : v.ny);
    const size_t n1 = static_cast<size_t>(axis == 0 ? v.ny : v.nx) + 2 * kSlabPad;
    return n0 * (static_cast<size_t>(v.nz) + 2 * kSlabPad) * n1;
}
cudaError_t launch_joseph_transpose(const float* vol, int nx, int ny, int nz,
    float* vol_yzx, float* vol_xzy, cudaStream_t s);
cudaError_t launch_joseph_fp(const float* slabs[3], const JosephView* views,
    const int* view_axis_host, int n_views, int nu, int nv, float* proj,
    int accumulate, cudaStream_t s);
cudaError_t launch_joseph_ray_table(const JosephView* views, int n_views,
    int nu, int nv, float4* rays, float* lens, cudaStream_t s);
// Iterative-solver vectors (iter_kernels.cu)
int dot_partial_count();
cudaError_t launch_dot_f64(const float* a, const float* b, size_t n, double* partials,
    double* result, cudaStream_t s);
cudaError_t launch_cgls_xr(const double* gamma, const double* ww, float* x, const float* p,
    size_t nx, float* r, const float* w, size_t nr, cudaStream_t s);
cudaError_t launch_cgls_p(const double* gamma_new, const double* gamma_old, float* p,
    const float* z, size_t n, cudaStream_t s);

// Siddon (siddon_kernels.cu); views in world coordinates
cudaError_t launch_siddon_fp(const float* vol, const ykb_cone_view* views, int n_views, int nu,
    int nv, const VolumeGrid& g, float* proj, int accumulate, cudaStream_t s);
cudaError_t launch_siddon_bp(const float* proj, const ykb_cone_view* views, int n_views, int nu,
    int nv, const VolumeGrid& g, float* vol, int accumulate, cudaStream_t s);
// (a1, e1) of every detector column from its first row into cols[n][nu];
// flag[0] = 1 when any ray of a column differs (the line backprojector
// then does not apply)
cudaError_t launch_joseph_column_table(const float4* rays, int n_views, int nu, int nv,
    float2* cols, int* flag, cudaStream_t s);
// matched backprojection for axial-column scans (see launch_joseph_column_table):
// weighted receives input x chord length per ray
cudaError_t launch_joseph_bp_lines(const float* proj, const float4* rays, const float* lens,
    const float2* cols, const float* view_proj, const JosephView* views, int n_views, int nu,
    int nv, const ykb_volume& vol, float* weighted, float* out, int accumulate, cudaStream_t s);
cudaError_t launch_joseph_bp(const float* proj, const float4* rays, const float* lens,
    const float* view_proj, const JosephView* views, int n_views, int nu, int nv,
    const ykb_volume& vol, float* weighted, float* out, int accumulate, cudaStream_t s);

} // namespace ykb

// Plan objects (opaque at the C-ABI).
struct ykb_fdk_plan {
    int device = 0;
    int n_views = 0, nu = 0, nv = 0;
    float scan_range = 0.f;
    ykb_volume volume{};
    ykb_filter filter{};
    int precision = YKB_PRECISION_FP32;
    bool axial = false;
    bool tc_filter = false;
    int tc_parts = 0;            // BF16 parts per operand of the tensor-core filter (2 or 3)
    int tc_near = 0;             // K chunks each side of a tile that its 2^-16 products cover
    int batch_capacity = 0;      // views the workspace holds
    int ld = 0;                  // row pitch (elements) of the filtered workspace
    int layout = 0;              // FilteredLayout of the filtered workspace
    int lda = 0;                 // row pitch of the bf16 GEMM operands (tensor-core filter)
    bool use_tma = false;        // TMA-staged backprojection
    int tma_bw = 0, tma_bh = 0;  // its projection box
    ykb::PipelineWait bp_wait;   // its pipeline-wait limit (tests shorten it)
    std::vector<ykb::FdkDerived> derived;
    ykb::DeviceBuffer coef;      // FdkViewCoef[n_views]
    ykb::DeviceBuffer pwv;       // FdkPreweightView[n_views]
    ykb::DeviceBuffer ramp;      // float[2*nu-1]
    ykb::DeviceBuffer parker;    // float[n_views][nu] short-scan weights, or empty
    ykb::DeviceBuffer toeplitz_hi, toeplitz_lo, toeplitz_lo2;  // bf16 [nu][lda] split parts
    ykb::DeviceBuffer work_a;    // preweighted rows: float, or the bf16 split parts in turn
    ykb::DeviceBuffer work_filtered;  // filtered projections (layout, pitch ld)
    ykb::DeviceBuffer err_flag;  // int[4]: device error word, box pre-pass scratch
    // stage timing (ykb_fdk_stage_timing): a start and a stop event around
    // each filter (stage 0) and backprojection (stage 1) launch group, on the
    // stream that launches it; events are pooled and reused
    struct StageEvents { cudaEvent_t start = nullptr, stop = nullptr; int stage = 0; };
    bool timing = false;
    std::vector<StageEvents> stage_events;
    size_t stage_events_used = 0;
    // tensor-core filter: the preweight of the next sub-batch of views runs on
    // this stream while the ramp filter of the current one runs on the
    // caller's (created on first use)
    static constexpr int kFilterSubBatches = 4;
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t aux_in = nullptr;                       // the caller's stream reached the filter
    cudaEvent_t aux_done[kFilterSubBatches] = {};       // sub-batch preweighted
    // host-input streaming (ykb_fdk_execute_host), created on first use
    ykb::DeviceBuffer stage_in;  // two batches of input views
    int stage_views = 0;         // views per batch slot
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr};    // batch slot filled
    cudaEvent_t consumed[2] = {nullptr, nullptr};  // batch slot read by the filter
    ~ykb_fdk_plan()
    {
        for (auto& e : stage_events) {
            if (e.start) cudaEventDestroy(e.start);
            if (e.stop) cudaEventDestroy(e.stop);
        }
        for (cudaEvent_t e : aux_done) if (e) cudaEventDestroy(e);
        if (aux_in) cudaEventDestroy(aux_in);
        if (aux_stream) cudaStreamDestroy(aux_stream);
        for (cudaEvent_t e : copied) if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : consumed) if (e) cudaEventDestroy(e);
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }
};

struct ykb_joseph_plan {
    int device = 0;
    int n_views = 0, nu = 0, nv = 0;
    ykb_volume volume{};
    std::vector<ykb::JosephView> host_views;
    std::vector<ykb_cone_view> cone_views;
    std::vector<int> axes;
    ykb::DeviceBuffer views;     // JosephView[n]
    ykb::DeviceBuffer view_proj; // float[n][12]: voxel-space 3x4 projection
    ykb::DeviceBuffer rays;      // float4[n*nv*nu]: (a1, e1, a2, e2)
    ykb::DeviceBuffer lens;      // float[n*nv*nu]: chord length per step
    // backprojector input x chord length: float[n*nv*nu], or for the column
    // backprojector float4 (a2, e2, input x chord length, 0)
    ykb::DeviceBuffer weighted;
    bool column_bp = false;      // every view's detector columns are axial (line backprojector)
    ykb::DeviceBuffer cols;      // float2[n*nu]: (a1, e1) per detector column
    ykb::DeviceBuffer slab_y, slab_x;  // transposed volume copies
    ykb::DeviceBuffer world_views;     // ykb_cone_view[n] (Siddon), uploaded on first use
    // pseudo-matched backprojection, set up on first use
    bool pseudo_ready = false;
    bool pseudo_axial = false;         // untilted detector: the axial column walk
    int pseudo_bw = 0, pseudo_bh = 0;  // TMA projection box (0: bounds-checked loads)
    int pseudo_ld = 0;                 // tap-pair row pitch
    ykb::DeviceBuffer fdk_coef;        // FdkViewCoef[n]
    ykb::DeviceBuffer pseudo_coef;     // PseudoViewCoef[n]
    ykb::DeviceBuffer pairs;           // projections as tap pairs [n][nv][pseudo_ld]
    ykb::DeviceBuffer err_flag;        // int[4]: device error word, box pre-pass scratch
};

struct ykb_iter {
    int device = 0;
    ykb::DeviceBuffer partials;  // double[dot_partial_count()]
};
