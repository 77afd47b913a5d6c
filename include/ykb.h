/*
 * ykb.h -- C-ABI of the B200-native flat-panel circular cone-beam FDK and
 * Joseph forward/back projector library (libykb.so).
 *
 * This is the boundary that replaces the reference's internal CUDA entry
 * points for the path; the C++ Session layer (include/ykb_session.hpp, same
 * names as YKCBCT's public YkReconstructionApi.hpp) and the torch extension
 * (fdk_cuda_impl_b200) both call it.  Every entry point:
 *   - takes plain pointers and sizes (device pointers unless stated),
 *   - is ordered on the caller's CUDA stream (cudaStream_t passed as
 *     ykb_stream) and does not synchronise unless stated,
 *   - never aborts and never throws; it returns a ykb_status whose values
 *     1..7 are the reference's YK::EApiErrorCode values
 *     (include/YKCBCT/interface/YkReconstructionApi.hpp:72-81) and
 *     ykb_last_error() returns the calling thread's last message.
 * Layouts are the reference's: projections [view][v][u] and volumes
 * [z][y][x], contiguous float32 (include/YKCBCT/interface/
 * YkReconstructionTypes.hpp:38-44; doc/geometry-and-data.md).
 */
#ifndef YKB_H
#define YKB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define YKB_API __declspec(dllexport)
#else
#define YKB_API __attribute__((visibility("default")))
#endif

typedef struct CUstream_st* ykb_stream; /* identical to cudaStream_t */

typedef struct { float x, y, z, w; } ykb_float4;

/* One view of flat cone-beam vector geometry; byte layout of
 * YK::SConeProjGeomVec (include/YKCBCT/geometry/YkProjectionGeometry.hpp:12-18):
 * pixel (u,v) centre = detS + u*detU + v*detV, angle.x = view angle (rad). */
typedef struct {
    ykb_float4 src;
    ykb_float4 detS;
    ykb_float4 detU;
    ykb_float4 detV;
    ykb_float4 angle;
} ykb_cone_view;

/* Volume grid; voxel (i,j,k) centre = center + (index - (n-1)/2) * vox,
 * as YK::SVolGeom::origin() (include/YKCBCT/geometry/YkVolumeGeometry.hpp:9-55). */
typedef struct {
    int nx, ny, nz;
    float vox_x, vox_y, vox_z;
    float center_x, center_y, center_z;
} ykb_volume;

/* Ramp filter selection; members and enum values of YK::SAnalyticFilterParams /
 * YK::EFdkFilter (include/YKCBCT/algorithms/analytic/YkAnalyticFilterParams.hpp:5-14). */
typedef struct {
    int type;      /* 0 None 1 RamLak 2 SheppLogan 3 Cosine 4 Hann 5 Hamming
                      6 Blackman 7 Butterworth 8 Kaiser 9 Tukey */
    float cutoff;  /* cycles/sample, (0, 0.5] */
    float gain;
    float butterworth_order;
    float kaiser_beta;
    float tukey_alpha;
} ykb_filter;

/* Regular circular orbit with a flat detector: YK::SRegularCircularScanSpec
 * and YK::SFlatDetectorSpec (include/YKCBCT/geometry/YkGeometryBuilderTypes.hpp). */
typedef struct {
    int total_views;
    int views_per_turn;
    float start_angle_rad;
    int rotation_direction; /* +1 / -1 */
    float sid_mm;
    float sdd_mm;
    float z_mm;
    float source_offset_mm[3];
    int channels;
    int rows;
    float channel_size_mm;
    float row_size_mm;
    float offset_unv_mm[3]; /* U, N, V */
    float tilt_u_rad;
    float tilt_v_rad;
    float tilt_n_rad;
} ykb_circular_flat;

typedef enum {
    YKB_OK = 0,
    YKB_ERR_INVALID_CONFIG = 1,    /* EApiErrorCode::InvalidConfig */
    YKB_ERR_INVALID_GEOMETRY = 2,  /* EApiErrorCode::InvalidGeometry */
    YKB_ERR_UNSUPPORTED = 3,       /* EApiErrorCode::UnsupportedCombination */
    YKB_ERR_INVALID_BUFFER = 5,    /* EApiErrorCode::InvalidBuffer */
    YKB_ERR_STREAMING_STATE = 6,   /* EApiErrorCode::StreamingStateError */
    YKB_ERR_CUDA = 7,              /* EApiErrorCode::CudaError */
    YKB_ERR_OUT_OF_MEMORY = 8
} ykb_status;

typedef enum {
    YKB_PRECISION_FP32 = 0, /* FP32 ramp filter */
    YKB_PRECISION_BF16 = 1  /* BF16 tensor-core (tcgen05) Toeplitz filter with
                               split hi/lo correction and FP32 accumulation;
                               pairs with BF16 projection input */
} ykb_precision;

typedef enum { YKB_DTYPE_F32 = 0, YKB_DTYPE_BF16 = 1 } ykb_dtype;

typedef struct ykb_fdk_plan ykb_fdk_plan;
typedef struct ykb_joseph_plan ykb_joseph_plan;

/* Library version (major*10000 + minor*100 + patch). */
YKB_API int ykb_version(void);

/* Message of the last failed call on the calling thread ("" if none). */
YKB_API const char* ykb_last_error(void);

/* Regular scan range 2*pi*total_views/views_per_turn in float, as
 * regularScanRangeRad (include/YKCBCT/interface/YkSystemReconstruction.hpp:22-28). */
YKB_API float ykb_regular_scan_range(int total_views, int views_per_turn);

/* Per-view flat geometry of a regular circular orbit; replaces
 * buildCircularTrajectory + buildProjectionGeometry
 * (include/YKCBCT/geometry/YkSystemGeometry.hpp:61-73,
 * include/YKCBCT/geometry/YkModularGeometryBuilder.hpp:9-17).  Host only;
 * out must hold spec->total_views entries (capacity). */
YKB_API ykb_status ykb_build_circular_flat(const ykb_circular_flat* spec,
    ykb_cone_view* out, int capacity);

/* ---------------------------------------------------------------- FDK --- */

/* Prepares an FDK plan for the full view sequence (host geometry, copied):
 * derived geometry in FP64, projection coefficients, ramp kernel, device
 * workspace.  Replaces FdkPipeline::prepareWithGeometry
 * (src/Reconstruction/Analytic/Circular/Flat/FDK/YkFdkPipeline.hpp:344-383).
 * scan_range_rad is the regular scan range (ykb_regular_scan_range). */
YKB_API ykb_status ykb_fdk_plan_create(const ykb_cone_view* views, int n_views,
    int nu, int nv, float scan_range_rad, const ykb_volume* volume,
    const ykb_filter* filter, int precision, int device, ykb_fdk_plan** plan);

/* Parker short-scan weighting (YK::EParkerMode values, include/YKCBCT/
 * algorithms/analytic/YkFdkParams.hpp): AUTO weights scans shorter than 2 pi. */
typedef enum {
    YKB_PARKER_AUTO = 0,
    YKB_PARKER_DISABLED = 1,
    YKB_PARKER_ENABLED = 2
} ykb_parker_mode;

/* ykb_fdk_plan_create with Parker weighting for short scans: views keep the
 * scan's start angle and rotation direction (+1/-1), from which each view's
 * position along the scan is measured.  Enabled (or Auto below 2 pi) on a
 * scan shorter than pi + 2 x fan angle, or on a full turn, is
 * YKB_ERR_INVALID_GEOMETRY, as the reference's prepare rejects it
 * (src/Reconstruction/Analytic/Circular/Flat/FDK/YkFdkPipeline.hpp:597-635).
 * The weights are those of .../FDK/kernels/YkFDKParkerKernels.cu:46-138,
 * applied between the cosine preweight and the ramp filter.
 * ykb_fdk_plan_create is this call with YKB_PARKER_DISABLED. */
YKB_API ykb_status ykb_fdk_plan_create_ex(const ykb_cone_view* views, int n_views,
    int nu, int nv, float scan_range_rad, float start_angle_rad,
    int rotation_direction, const ykb_volume* volume, const ykb_filter* filter,
    int precision, int parker_mode, int device, ykb_fdk_plan** plan);

YKB_API ykb_status ykb_fdk_plan_destroy(ykb_fdk_plan* plan);

/* Cosine preweight + ramp filter + weighted backprojection of views
 * [view_offset, view_offset+n_views) of d_proj ([n_views][nv][nu], dtype
 * proj_dtype) into d_volume ([nz][ny][nx] float).  clear_output=1 zeroes the
 * volume first, else the batch accumulates (streaming FDK).  Replaces
 * FdkPipeline::enqueueBatch (YkFdkPipeline.hpp:388-488). */
YKB_API ykb_status ykb_fdk_execute(ykb_fdk_plan* plan, const void* d_proj,
    int proj_dtype, int view_offset, int n_views, float* d_volume,
    int clear_output, ykb_stream stream);

/* The same FDK with the projections in HOST memory: the views are copied
 * to the device in batches on an internal copy stream, double-buffered, so
 * that the copy of batch b+1 overlaps the filter and backprojection of
 * batch b on `stream`.  Pinned (page-locked) h_proj gives full overlap; a
 * pageable buffer works but each batch copy first passes through the
 * driver's staging on the calling thread.  Returns once the work is
 * enqueued; h_proj must stay valid and unchanged until `stream` has
 * completed it.  Replaces the host-projection path of FdkPipeline::enqueueBatch
 * (YkFdkPipeline.hpp:388-488, chunk uploads :454-457), which copies each
 * 32-view chunk synchronously in between its kernels. */
YKB_API ykb_status ykb_fdk_execute_host(ykb_fdk_plan* plan, const void* h_proj,
    int proj_dtype, int view_offset, int n_views, float* d_volume,
    int clear_output, ykb_stream stream);

/* ykb_fdk_execute_host with the volume returned to host memory as well:
 * the reconstruction accumulates in d_volume (device, [nz][ny][nx]) and is
 * copied to h_volume (host; pin it for the copies to overlap).  The last
 * projection batch is backprojected in z slabs and each finished slab is
 * copied behind the next slab's kernel, so most of the volume download
 * overlaps the GPU work.  Asynchronous on `stream`: the host volume is
 * complete when the stream's work up to this call has run.  Replaces the
 * Session's host-buffer FDK path (projection upload, FdkPipeline batches,
 * volume download; src/interface/YkSession.cpp:693-728). */
YKB_API ykb_status ykb_fdk_execute_host_out(ykb_fdk_plan* plan, const void* h_proj,
    int proj_dtype, int view_offset, int n_views, float* d_volume, float* h_volume,
    int clear_output, ykb_stream stream);

/* Stage entry: preweight + ramp filter only; d_filtered receives
 * [n_views][nv][nu] float.  Replaces PreweightProcessor::apply +
 * FilterProcessor::apply (.../FDK/YkFDKPreWeightProcessor.hpp,
 * .../FDK/YkFDKFilterProcessor.hpp:84-122). */
YKB_API ykb_status ykb_fdk_filter(ykb_fdk_plan* plan, const void* d_proj,
    int proj_dtype, int view_offset, int n_views, void* d_filtered,
    ykb_stream stream);

/* Stage entry: weighted backprojection of already filtered projections
 * (dtype filtered_dtype).  Replaces BpProcessor::apply / fdk_bp_kernel
 * (.../FDK/YkBackProjectProcessor.hpp:53-67,
 * .../FDK/kernels/YkFDKBpKernels.cu:112-209,336-381). */
YKB_API ykb_status ykb_fdk_backproject(ykb_fdk_plan* plan,
    const void* d_filtered, int filtered_dtype, int view_offset, int n_views,
    float* d_volume, int clear_output, ykb_stream stream);

/* Bytes of device workspace the plan holds (introspection). */
YKB_API size_t ykb_fdk_workspace_bytes(const ykb_fdk_plan* plan);

/* Synchronises `stream` and reports (then clears) the plan's device-side
 * error word: YKB_ERR_CUDA when a bounded pipeline wait timed out or a voxel
 * column fell outside its staged projection box (the kernels never hang or
 * fault on these; they stop and record them).  The reference has no
 * equivalent: it aborts the process on CUDA errors (src/global/YkMacro.hpp:35-41). */
YKB_API ykb_status ykb_fdk_check(ykb_fdk_plan* plan, ykb_stream stream);

/* Stage timing: while enabled, the plan records a CUDA event pair around
 * each filter launch group (cosine preweight + ramp filter of one workspace
 * chunk) and each backprojection launch group, on the stream that launches
 * it.  ykb_fdk_stage_times synchronises `stream`, returns the summed event
 * times (ms) and group counts of each stage since the last call (or since
 * timing was enabled) and starts a new tally.  For measurement: the stages'
 * own device times inside a full execute.  No counterpart in the
 * reference. */
YKB_API ykb_status ykb_fdk_stage_timing(ykb_fdk_plan* plan, int enable);
YKB_API ykb_status ykb_fdk_stage_times(ykb_fdk_plan* plan, ykb_stream stream,
    double* filter_ms, int* filter_groups, double* backproject_ms,
    int* backproject_groups);

/* Test hook for the timeout path of the TMA backprojection: sets the limit
 * of its pipeline waits to wait_ns (0 restores the default, about 2 s) and,
 * when withheld_view >= 0, makes the copy producer skip that view (an index
 * within each backprojection launch) so that every wait for it runs out.  A
 * wait that runs out sets the plan's error word, which ykb_fdk_check
 * reports; the kernel ends without hanging, its copies in flight drained, and
 * the plan stays usable (call again with 0, -1 to restore).  Waits that drain
 * copies keep the default limit.  No counterpart in the reference. */
YKB_API ykb_status ykb_fdk_test_pipeline_wait(ykb_fdk_plan* plan,
    unsigned long long wait_ns, int withheld_view);

/* The preweight + ramp filter stage of ykb_fdk_filter for callers that
 * cannot call cudaMalloc (an application whose memory pool owns the GPU,
 * a real-time loop that forbids allocation after start-up): no plan and no
 * device allocation.  This entry point has no counterpart in the reference.
 * Geometry and filter come from the host arguments (as ykb_fdk_plan_create
 * takes them); d_proj holds [n_views][nv][nu] (proj_dtype), d_filtered
 * receives [n_views][nv][nu] float.  Full scans only (scan_range_rad >=
 * 2 pi): a short scan needs Parker weights, which only a plan applies, and
 * returns YKB_ERR_INVALID_CONFIG.  Scratch is one fixed 32 MiB device array
 * inside the library, present on every GPU that loads it until exit;
 * limits: nu <= 8192, n_views <= 16384, nu*nv*4 <= 30,867,456 bytes
 * (29.4 MiB) per view, else YKB_ERR_INVALID_CONFIG.  The first call on a
 * device looks up that device's scratch address (cudaGetSymbolAddress).
 * All calls share the one array: calls that overlap on the GPU
 * (different streams, without ordering between them) race and corrupt each
 * other. */
YKB_API ykb_status ykb_fdk_filter_static(const ykb_cone_view* views,
    int n_views, int nu, int nv, float scan_range_rad, const ykb_filter* filter,
    const void* d_proj, int proj_dtype, float* d_filtered, ykb_stream stream);

/* ------------------------------------------------------------- Joseph --- */

/* Prepares the Joseph projector pair for a view sequence.  Replaces
 * ForwardOperator/BackOperator::prepare for FP_Joseph/BP_Joseph
 * (src/common/YkProjectionOperators.hpp:120-135,229-240). */
YKB_API ykb_status ykb_joseph_plan_create(const ykb_cone_view* views,
    int n_views, int nu, int nv, const ykb_volume* volume, int device,
    ykb_joseph_plan** plan);

YKB_API ykb_status ykb_joseph_plan_destroy(ykb_joseph_plan* plan);

/* d_proj ([n][nv][nu]) = (accumulate ? d_proj : 0) + A d_volume.  Replaces
 * ForwardOperator::apply with FP_Joseph (src/common/YkProjectionOperators.hpp:
 * 138-180) and fp_joseph_launch (src/FlatFpBp/FP/kernels/YkFPKernels.cu:530-565). */
YKB_API ykb_status ykb_joseph_fp(ykb_joseph_plan* plan, const float* d_volume,
    float* d_proj, int accumulate, ykb_stream stream);

/* d_volume = (accumulate ? d_volume : 0) + A^T d_proj, the exact transpose of
 * ykb_joseph_fp, computed voxel-driven without atomics.  Replaces
 * BackOperator::apply with BP_Joseph (src/common/YkProjectionOperators.hpp:
 * 293-298) and joseph_bp_launch (src/FlatFpBp/BP/kernels/YkBPJosephKernel.cu:
 * 226-266). */
YKB_API ykb_status ykb_joseph_bp(ykb_joseph_plan* plan, const float* d_proj,
    float* d_volume, int accumulate, ykb_stream stream);

/* Operator tasks of a projector plan: the values of YK::ETask
 * (src/common/YkOperatorTypes.hpp:5-22) that this library implements. */
typedef enum ykb_task {
    YKB_TASK_FP_JOSEPH = 1,
    YKB_TASK_FP_SIDDON = 2,
    YKB_TASK_BP_SIDDON_RAY_DRIVEN = 4,
    YKB_TASK_BP_FDK_PSEUDO_MATCHED = 7,
    YKB_TASK_BP_JOSEPH = 8
} ykb_task;

/* Applies one operator of the plan's view sequence.  Forward tasks read a
 * volume [nz][ny][nx] from d_in and write projections [n][nv][nu] to d_out,
 * back tasks the reverse; d_out = (accumulate ? d_out : 0) + op(d_in).
 * Replaces IForwardOperator/IBackOperator::apply for the task
 * (src/common/YkProjectionOperators.hpp:138-180,242-340).
 *   YKB_TASK_FP_JOSEPH, YKB_TASK_BP_JOSEPH: ykb_joseph_fp, ykb_joseph_bp.
 *   YKB_TASK_FP_SIDDON, YKB_TASK_BP_SIDDON_RAY_DRIVEN: the Siddon pair,
 *     exact intersection lengths of the source-to-pixel-centre ray with each
 *     voxel (fp_siddon_launch, src/FlatFpBp/FP/kernels/YkFPSiddonKernel.cu:
 *     19-129,283-316; bp_siddon_launch, src/FlatFpBp/BP/kernels/
 *     YkBPSiddonKernel.cu:31-160).  The backprojector is the exact transpose
 *     of the projector; it sums with global atomics, so its last bits vary
 *     between runs.
 *   YKB_TASK_BP_FDK_PSEUDO_MATCHED: voxel-driven bilinear backprojection
 *     with the weight L^3 / (|P - S|^2 SDD_plane) x voxel volume / pixel
 *     area (fdk_pseudo_matched_bp_launch, src/FlatFpBp/BP/kernels/
 *     YkBpFdkKernel.cu:356-450,532-548), an approximate transpose of the
 *     forward projector.  Its first call builds the plan's tables for it
 *     (synchronising the stream) and a tap-pair copy of the projections
 *     (8 bytes per pixel).
 * Other task values return YKB_ERR_UNSUPPORTED. */
YKB_API ykb_status ykb_operator_apply(ykb_joseph_plan* plan, int task,
    const float* d_in, float* d_out, int accumulate, ykb_stream stream);

/* Reads and clears the plan's device error word (pseudo-matched
 * backprojection); synchronises the stream.  YKB_ERR_CUDA with the reasons
 * when it was set. */
YKB_API ykb_status ykb_joseph_check(ykb_joseph_plan* plan, ykb_stream stream);

/* Bytes of device workspace the plan holds (introspection). */
YKB_API size_t ykb_joseph_workspace_bytes(const ykb_joseph_plan* plan);

/* ------------------------------------------------- iterative solvers --- */

/* Vector kernels for the solvers that drive the projector pair (CGLS,
 * src/Reconstruction/Iterative/Flat/YkCglsBackends.hpp:70-150).  A context
 * holds the reduction workspace of one device; calls on one context from
 * streams without ordering between them race on it. */
typedef struct ykb_iter ykb_iter;
YKB_API ykb_status ykb_iter_create(int device, ykb_iter** ctx);
YKB_API ykb_status ykb_iter_destroy(ykb_iter* ctx);

/* *d_result = sum a[i] b[i] accumulated in FP64, deterministic, written on
 * the device (no host synchronisation).  Replaces dot_launch
 * (src/Reconstruction/Iterative/Common/kernels/YkIterKernels.cu:367-430),
 * which reduces in FP32 and returns through the host. */
YKB_API ykb_status ykb_dot_f64(ykb_iter* ctx, const float* d_a, const float* d_b, size_t n,
    double* d_result, ykb_stream stream);

/* CGLS updates with device-resident step sizes:
 *   ykb_cgls_update_xr: x += a p, r -= a w with a = *d_gamma / *d_ww
 *   ykb_cgls_update_p:  p = z + b p with b = *d_gamma_new / *d_gamma_old
 * (a ratio with a zero denominator counts as 0). */
YKB_API ykb_status ykb_cgls_update_xr(ykb_iter* ctx, const double* d_gamma, const double* d_ww,
    float* d_x, const float* d_p, size_t nx, float* d_r, const float* d_w, size_t nr,
    ykb_stream stream);
YKB_API ykb_status ykb_cgls_update_p(ykb_iter* ctx, const double* d_gamma_new,
    const double* d_gamma_old, float* d_p, const float* d_z, size_t n, ykb_stream stream);

/* ----------------------------------------------------------- diagnostics --- */

/* Measures the shared-memory load bandwidth of `device` (GB/s over all its
 * SMs): 4 CTAs per SM stream 16 KB of shared memory with conflict-free
 * vector loads of bytes_per_lane (8 or 16) bytes, best of five timed
 * launches (CUDA events) after one warm-up.  The on-chip peak that the
 * backprojection's two 8-byte tap-pair loads per voxel update are reported
 * against.  Synchronous; no counterpart in the reference. */
YKB_API ykb_status ykb_measure_shared_load_gbs(int device, int bytes_per_lane, double* gbs);

#ifdef __cplusplus
}
#endif

#endif /* YKB_H */
