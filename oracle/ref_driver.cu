// ref_driver.cu -- TEST INFRASTRUCTURE ONLY.  A thin extern "C" driver over
// the reference YKCBCT CUDA implementation, compiled from the reference's own
// sources (oracle/ref_build.py) into oracle/_ref/libykref.so.  It lets the
// parity tests compare libykb against the reference's actual outputs on the
// same inputs, and times the reference's device-resident FDK pipeline and
// Joseph operators on the same GPU.  Nothing in the product links it.
//
// The driver calls the reference's stock internal paths, the same ones its
// Session uses:
//   FDK     FdkPipeline::prepare(SSystemConfig, SReconstructionSpec, 32, ...)
//           then enqueueBatch / processBatchSync
//           (src/Reconstruction/Analytic/Circular/Flat/FDK/YkFdkPipeline.hpp:247-273,388-510;
//            the Session's own call is src/interface/YkSession.cpp:155-165,693-728)
//   FP      makeForwardOperator(ETask::FP_Joseph)->apply over a PreparedGeometry
//           built from the SSystemConfig (src/common/YkProjectionOperators.hpp:120-180,
//           src/common/YkExecutionContext.hpp:19-88)
//   BP      makeBackOperator(ETask::BP_Joseph)->apply (YkProjectionOperators.hpp:218-298)
//
// Geometry, volume and filter arrive in libykb's C-ABI structs (ykb.h), whose
// fields are those of the reference's SRegularCircularScanSpec,
// SFlatDetectorSpec, SVolumeGridSpec and SAnalyticFilterParams.
//
// The reference aborts the process on a CUDA error (src/global/YkMacro.hpp:35-41);
// callers run it in a child process.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "Reconstruction/Analytic/Circular/Flat/FDK/YkFdkPipeline.hpp"
#include "Reconstruction/Iterative/Flat/YkCglsBackends.hpp"
#include "common/YkExecutionContext.hpp"
#include "common/YkOperatorTypes.hpp"
#include "common/YkProjectionOperators.hpp"

#include "ykb.h"

namespace {

std::string g_error;

int fail(const char* what)
{
    g_error = what;
    return 1;
}

YK::SSystemConfig make_system(const ykb_circular_flat& s, const ykb_volume& v)
{
    YK::SSystemConfig sys{};
    sys.detector = YK::EDetectorKind::Flat;
    sys.trajectory = YK::ETrajectoryKind::Circular;
    sys.circular.total_views = s.total_views;
    sys.circular.views_per_turn = s.views_per_turn;
    sys.circular.start_angle_rad = s.start_angle_rad;
    sys.circular.rotation_direction = s.rotation_direction;
    sys.circular.sid_mm = s.sid_mm;
    sys.circular.sdd_mm = s.sdd_mm;
    sys.circular.z_mm = s.z_mm;
    sys.circular.source_offset_mm = make_float3(s.source_offset_mm[0], s.source_offset_mm[1],
        s.source_offset_mm[2]);
    sys.flat_detector.channels = s.channels;
    sys.flat_detector.rows = s.rows;
    sys.flat_detector.channel_size_mm = s.channel_size_mm;
    sys.flat_detector.row_size_mm = s.row_size_mm;
    sys.flat_detector.pose.offset_unv_mm = make_float3(s.offset_unv_mm[0], s.offset_unv_mm[1],
        s.offset_unv_mm[2]);
    sys.flat_detector.pose.tilt_u_rad = s.tilt_u_rad;
    sys.flat_detector.pose.tilt_v_rad = s.tilt_v_rad;
    sys.flat_detector.pose.tilt_n_rad = s.tilt_n_rad;
    sys.volume.nx = v.nx;
    sys.volume.ny = v.ny;
    sys.volume.nz = v.nz;
    sys.volume.voxel_x_mm = v.vox_x;
    sys.volume.voxel_y_mm = v.vox_y;
    sys.volume.voxel_z_mm = v.vox_z;
    sys.volume.center_mm = make_float3(v.center_x, v.center_y, v.center_z);
    return sys;
}

YK::SReconstructionSpec make_fdk_spec(const ykb_filter& f)
{
    YK::SReconstructionSpec r{};
    r.pipeline = YK::EPipeline::FDK;
    r.fdk.parker.mode = YK::EParkerMode::Auto;
    r.fdk.filter.type = static_cast<YK::EFdkFilter>(f.type);
    r.fdk.filter.cutoff = f.cutoff;
    r.fdk.filter.gain = f.gain;
    r.fdk.filter.butterworth_order = f.butterworth_order;
    r.fdk.filter.kaiser_beta = f.kaiser_beta;
    r.fdk.filter.tukey_alpha = f.tukey_alpha;
    return r;
}

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking); }
    ~Stream() { if (s) cudaStreamDestroy(s); }
};

template <class T>
struct Dev {
    T* p = nullptr;
    explicit Dev(size_t n) { if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) p = nullptr; }
    ~Dev() { if (p) cudaFree(p); }
};

float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

} // namespace

extern "C" {

__attribute__((visibility("default"))) const char* ykref_last_error() { return g_error.c_str(); }

// Full FDK of host projections [view][v][u] into a host volume [z][y][x],
// submitted in batches of `batch_views` views (0 = one batch).
__attribute__((visibility("default"))) int ykref_fdk(const ykb_circular_flat* scan,
    const ykb_volume* volume, const ykb_filter* filter, const float* h_proj, float* h_vol,
    int batch_views, int device)
{
    if (!scan || !volume || !filter || !h_proj || !h_vol) return fail("null argument");
    if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice");
    const YK::SSystemConfig sys = make_system(*scan, *volume);
    const YK::SReconstructionSpec spec = make_fdk_spec(*filter);
    Stream stream;
    YK::FdkPipeline fdk;
    if (!fdk.prepare(sys, spec, YK::kMaxChunkAng, stream.s, device)) return fail("FdkPipeline::prepare");
    const size_t nvox = size_t(volume->nx) * volume->ny * volume->nz;
    Dev<float> d_vol(nvox);
    if (!d_vol.p) return fail("cudaMalloc volume");
    const size_t view_elems = size_t(scan->channels) * scan->rows;
    const int total = scan->total_views;
    const int step = batch_views > 0 ? batch_views : total;
    for (int off = 0; off < total; off += step) {
        YK::FdkProjectionBatch b{};
        b.projection = h_proj + view_elems * off;
        b.count = std::min(step, total - off);
        b.location = YK::EMemoryLocation::Host;
        if (!fdk.processBatchSync(b, d_vol.p, off == 0)) return fail("FdkPipeline::processBatchSync");
    }
    if (cudaMemcpy(h_vol, d_vol.p, nvox * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail("cudaMemcpy volume");
    fdk.release();
    return 0;
}

// Full FDK as ykref_fdk in one batch, then reads back the pipeline's stage
// buffers of its last chunk (FdkPipeline::lastStage(), YkFdkPipeline.hpp:182-192,549):
// preweighted and filtered rows of views [*first_view, *first_view + *count).
// h_preweighted / h_filtered hold kMaxChunkAng views.
__attribute__((visibility("default"))) int ykref_fdk_stages(const ykb_circular_flat* scan,
    const ykb_volume* volume, const ykb_filter* filter, const float* h_proj, float* h_vol,
    float* h_preweighted, float* h_filtered, int* first_view, int* count, int device)
{
    if (!scan || !volume || !filter || !h_proj || !h_vol || !h_preweighted || !h_filtered ||
        !first_view || !count)
        return fail("null argument");
    if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice");
    const YK::SSystemConfig sys = make_system(*scan, *volume);
    const YK::SReconstructionSpec spec = make_fdk_spec(*filter);
    Stream stream;
    YK::FdkPipeline fdk;
    if (!fdk.prepare(sys, spec, YK::kMaxChunkAng, stream.s, device)) return fail("FdkPipeline::prepare");
    const size_t nvox = size_t(volume->nx) * volume->ny * volume->nz;
    Dev<float> d_vol(nvox);
    if (!d_vol.p) return fail("cudaMalloc volume");
    YK::FdkProjectionBatch b{};
    b.projection = h_proj;
    b.count = scan->total_views;
    b.location = YK::EMemoryLocation::Host;
    if (!fdk.processBatchSync(b, d_vol.p, true)) return fail("FdkPipeline::processBatchSync");
    const YK::FdkStageView& st = fdk.lastStage();
    if (!st.valid() || st.count > YK::kMaxChunkAng) return fail("no stage view");
    const size_t n = size_t(st.count) * scan->channels * scan->rows;
    if (cudaMemcpy(h_preweighted, st.d_preweighted, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(h_filtered, st.d_filtered, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(h_vol, d_vol.p, nvox * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail("cudaMemcpy stages");
    *first_view = st.first_view;
    *count = st.count;
    fdk.release();
    return 0;
}

// Times the reference FDK pipeline over `reps` full sequences after `warmup`.
// ms[0]: device-resident projections (DeviceToDevice chunk uploads inside the
// pipeline), volume on the device.  ms[1]: host projections, as the Session
// requires (src/interface/YkSession.cpp:702-707), plus the volume read back
// to the host.  The host projections and volume live in pinned memory
// (cudaMallocHost; the input is copied there before timing), the same kind
// of host memory the timed end-to-end path of libykb gets.  Both are
// CUDA-event times on the pipeline's stream, averaged per sequence.
// h_vol_out (optional) receives the volume of the last device-resident run.
__attribute__((visibility("default"))) int ykref_fdk_time(const ykb_circular_flat* scan,
    const ykb_volume* volume, const ykb_filter* filter, const float* h_proj, int warmup, int reps,
    float* ms, float* h_vol_out, int device)
{
    if (!scan || !volume || !filter || !h_proj || !ms || reps <= 0) return fail("bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice");
    const YK::SSystemConfig sys = make_system(*scan, *volume);
    const YK::SReconstructionSpec spec = make_fdk_spec(*filter);
    Stream stream;
    YK::FdkPipeline fdk;
    if (!fdk.prepare(sys, spec, YK::kMaxChunkAng, stream.s, device)) return fail("FdkPipeline::prepare");
    const size_t nvox = size_t(volume->nx) * volume->ny * volume->nz;
    const size_t nproj = size_t(scan->channels) * scan->rows * scan->total_views;
    Dev<float> d_vol(nvox), d_proj(nproj);
    if (!d_vol.p || !d_proj.p) return fail("cudaMalloc");
    struct Pinned {
        float* p = nullptr;
        explicit Pinned(size_t n) { if (cudaMallocHost(&p, n * sizeof(float)) != cudaSuccess) p = nullptr; }
        ~Pinned() { if (p) cudaFreeHost(p); }
    } pin_proj(nproj), pin_vol(nvox);
    if (!pin_proj.p || !pin_vol.p) return fail("cudaMallocHost");
    std::memcpy(pin_proj.p, h_proj, nproj * sizeof(float));
    if (cudaMemcpy(d_proj.p, pin_proj.p, nproj * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail("cudaMemcpy projections");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto run = [&](bool device_input) {
        fdk.reset();
        YK::FdkProjectionBatch b{};
        b.projection = device_input ? d_proj.p : pin_proj.p;
        b.count = scan->total_views;
        b.location = device_input ? YK::EMemoryLocation::Device : YK::EMemoryLocation::Host;
        if (!fdk.processBatch(b, d_vol.p, true)) return false;
        if (!device_input)
            cudaMemcpyAsync(pin_vol.p, d_vol.p, nvox * sizeof(float), cudaMemcpyDeviceToHost, stream.s);
        return true;
    };
    for (int mode = 0; mode < 2; ++mode) {
        const bool device_input = mode == 0;
        for (int i = 0; i < warmup; ++i)
            if (!run(device_input)) return fail("FdkPipeline::processBatch");
        cudaStreamSynchronize(stream.s);
        cudaEventRecord(e0, stream.s);
        for (int i = 0; i < reps; ++i)
            if (!run(device_input)) return fail("FdkPipeline::processBatch");
        cudaEventRecord(e1, stream.s);
        if (cudaEventSynchronize(e1) != cudaSuccess) return fail("cudaEventSynchronize");
        ms[mode] = elapsed(e0, e1) / reps;
        if (device_input && h_vol_out &&
            cudaMemcpy(h_vol_out, d_vol.p, nvox * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail("cudaMemcpy volume");
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    fdk.release();
    return 0;
}

namespace {

// mode 0: FP_Joseph volume -> projections; mode 1: BP_Joseph projections -> volume.
int joseph(int mode, const ykb_circular_flat* scan, const ykb_volume* volume, const float* h_in,
    float* h_out, int warmup, int reps, float* ms, int device)
{
    if (!scan || !volume || !h_in || !h_out) return fail("null argument");
    if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice");
    const YK::SSystemConfig sys = make_system(*scan, *volume);
    YK::PreparedGeometry geometry;
    if (!geometry.initialize(sys)) return fail("PreparedGeometry::initialize");
    Stream stream;
    YK::ResourceContext resources;
    resources.attach(stream.s, device);
    const size_t nvox = size_t(volume->nx) * volume->ny * volume->nz;
    const size_t nproj = size_t(scan->channels) * scan->rows * scan->total_views;
    // mode: 0 FP_Joseph, 1 BP_Joseph, 2 BP_FDK_PseudoMatched, 3 FP_Siddon,
    // 4 BP_Siddon_RayDriven
    const bool forward = mode == 0 || mode == 3;
    const size_t n_in = forward ? nvox : nproj, n_out = forward ? nproj : nvox;
    Dev<float> d_in(n_in), d_out(n_out);
    if (!d_in.p || !d_out.p) return fail("cudaMalloc");
    if (cudaMemcpy(d_in.p, h_in, n_in * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail("cudaMemcpy input");
    std::unique_ptr<YK::IForwardOperator> fp;
    std::unique_ptr<YK::IBackOperator> bp;
    if (forward) {
        fp = YK::makeForwardOperator(mode == 3 ? YK::ETask::FP_Siddon : YK::ETask::FP_Joseph);
        if (!fp->prepare(geometry, resources)) return fail("ForwardOperator::prepare");
    } else {
        bp = YK::makeBackOperator(mode == 2 ? YK::ETask::BP_FDK_PseudoMatched
            : mode == 4 ? YK::ETask::BP_Siddon_RayDriven : YK::ETask::BP_Joseph);
        if (!bp->prepare(geometry, resources)) return fail("BackOperator::prepare");
    }
    auto apply = [&]() {
        return forward ? fp->apply(d_in.p, geometry.base(), d_out.p, resources)
                       : bp->apply(d_in.p, geometry.base(), d_out.p, true, resources);
    };
    if (!apply()) return fail("operator apply");
    if (cudaStreamSynchronize(stream.s) != cudaSuccess) return fail("operator execution");
    if (cudaMemcpy(h_out, d_out.p, n_out * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail("cudaMemcpy output");
    if (ms && reps > 0) {
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        for (int i = 0; i < warmup; ++i) apply();
        cudaStreamSynchronize(stream.s);
        cudaEventRecord(e0, stream.s);
        for (int i = 0; i < reps; ++i) apply();
        cudaEventRecord(e1, stream.s);
        if (cudaEventSynchronize(e1) != cudaSuccess) return fail("cudaEventSynchronize");
        *ms = elapsed(e0, e1) / reps;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (fp) fp->release();
    if (bp) bp->release();
    return 0;
}

} // namespace

// The reference's CGLS (CglsAstraBackend, src/Reconstruction/Iterative/Flat/
// YkCglsBackends.hpp:22-196) for n_iter iterations from a zero volume, with
// FP_Joseph and, per `matched`, BP_Joseph (1) or its default
// BP_FDK_PseudoMatched (0).  ms (optional) receives the device time of run().
__attribute__((visibility("default"))) int ykref_cgls(const ykb_circular_flat* scan,
    const ykb_volume* volume, const float* h_proj, float* h_vol, int n_iter, int matched,
    float* ms, int device)
{
    if (!scan || !volume || !h_proj || !h_vol || n_iter <= 0) return fail("bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice");
    const YK::SSystemConfig sys = make_system(*scan, *volume);
    YK::PreparedGeometry geometry;
    if (!geometry.initialize(sys)) return fail("PreparedGeometry::initialize");
    Stream stream;
    const size_t nvox = size_t(volume->nx) * volume->ny * volume->nz;
    const size_t nproj = size_t(scan->channels) * scan->rows * scan->total_views;
    Dev<float> d_proj(nproj), d_vol(nvox);
    if (!d_proj.p || !d_vol.p) return fail("cudaMalloc");
    if (cudaMemcpy(d_proj.p, h_proj, nproj * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(d_vol.p, 0, nvox * sizeof(float)) != cudaSuccess)
        return fail("upload");
    YK::CglsAstraBackend cgls;
    YK::CglsAstraBackend::Config cfg{};
    cfg.n_iter = n_iter;
    cfg.fp_task = YK::ETask::FP_Joseph;
    cfg.bp_task = matched ? YK::ETask::BP_Joseph : YK::ETask::BP_FDK_PseudoMatched;
    if (!cgls.init(geometry.base(), cfg, geometry.allGeometry(), stream.s, device))
        return fail("CglsAstraBackend::init");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream.s);
    const bool ok = cgls.run(d_proj.p, d_vol.p, geometry.base(), stream.s);
    cudaEventRecord(e1, stream.s);
    cudaEventSynchronize(e1);
    if (ms) *ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok) return fail("CglsAstraBackend::run");
    if (cudaMemcpy(h_vol, d_vol.p, nvox * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail("download");
    cgls.release();
    return 0;
}

// Joseph forward projection (FP_Joseph) of a host volume; optional timing
// (ms != NULL, reps > 0) of the operator call on the device-resident volume.
__attribute__((visibility("default"))) int ykref_joseph_fp(const ykb_circular_flat* scan,
    const ykb_volume* volume, const float* h_vol, float* h_proj, int warmup, int reps, float* ms,
    int device)
{
    return joseph(0, scan, volume, h_vol, h_proj, warmup, reps, ms, device);
}

// Joseph backprojection (BP_Joseph, clear_volume) of host projections.
__attribute__((visibility("default"))) int ykref_joseph_bp(const ykb_circular_flat* scan,
    const ykb_volume* volume, const float* h_proj, float* h_vol, int warmup, int reps, float* ms,
    int device)
{
    return joseph(1, scan, volume, h_proj, h_vol, warmup, reps, ms, device);
}

// ForwardOperator with FP_Siddon and BackOperator with BP_Siddon_RayDriven
// (src/common/YkProjectionOperators.hpp:159-171,262-270); arguments as
// ykref_joseph_fp / ykref_joseph_bp.
__attribute__((visibility("default"))) int ykref_siddon_fp(const ykb_circular_flat* scan,
    const ykb_volume* volume, const float* h_vol, float* h_proj, int warmup, int reps, float* ms,
    int device)
{
    return joseph(3, scan, volume, h_vol, h_proj, warmup, reps, ms, device);
}

__attribute__((visibility("default"))) int ykref_siddon_bp(const ykb_circular_flat* scan,
    const ykb_volume* volume, const float* h_proj, float* h_vol, int warmup, int reps, float* ms,
    int device)
{
    return joseph(4, scan, volume, h_proj, h_vol, warmup, reps, ms, device);
}

// BackOperator with BP_FDK_PseudoMatched (src/common/YkProjectionOperators.hpp:
// 324-333), clear volume; arguments as ykref_joseph_bp.
__attribute__((visibility("default"))) int ykref_bp_pseudo(const ykb_circular_flat* scan,
    const ykb_volume* volume, const float* h_proj, float* h_vol, int warmup, int reps, float* ms,
    int device)
{
    return joseph(2, scan, volume, h_proj, h_vol, warmup, reps, ms, device);
}

} // extern "C"
