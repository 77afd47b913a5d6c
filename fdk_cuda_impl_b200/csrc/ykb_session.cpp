// C++ Session layer over the C-ABI (include/ykb_session.hpp).  Validation
// order, error codes and streaming rules follow ReconstructionSession
// (src/interface/YkReconstructionApi.cpp:137-397) and Session::executeFdk_ /
// executeFp_ (src/interface/YkSession.cpp:693-728, 881-939).
#include "ykb_session.hpp"
#include "ykb_internal.hpp"

#include <cmath>
#include <cstddef>
#include <new>
#include <string>
#include <vector>

namespace YK {
namespace {

bool has_bytes(uint32_t actual, size_t required) { return actual >= required; }

bool valid_location(EMemoryLocation l) { return l == EMemoryLocation::Host || l == EMemoryLocation::Device; }

static_assert(sizeof(SConeProjGeomVec) == sizeof(ykb_cone_view), "view layout");

ykb_cone_view to_view(const SConeProjGeomVec& f)
{
    auto c = [](const float4& v) { return ykb_float4{v.x, v.y, v.z, v.w}; };
    return ykb_cone_view{c(f.src), c(f.detS), c(f.detU), c(f.detV), c(f.angle)};
}

// Caller frames for forward projection: finite source and detector vectors,
// detU and detV orthogonal to 1e-5 and a finite angle (PreparedGeometry::
// initialize, src/common/YkExecutionContext.hpp:23-38)
bool valid_frame(const SConeProjGeomVec& f)
{
    for (const float4& a : {f.src, f.detS, f.detU, f.detV})
        if (!std::isfinite(a.x) || !std::isfinite(a.y) || !std::isfinite(a.z)) return false;
    const double uu = double(f.detU.x) * f.detU.x + double(f.detU.y) * f.detU.y + double(f.detU.z) * f.detU.z;
    const double vv = double(f.detV.x) * f.detV.x + double(f.detV.y) * f.detV.y + double(f.detV.z) * f.detV.z;
    const double uv = double(f.detU.x) * f.detV.x + double(f.detU.y) * f.detV.y + double(f.detU.z) * f.detV.z;
    return uu > 0 && vv > 0 && std::abs(uv) <= 1e-5 * std::sqrt(uu * vv) && std::isfinite(f.angle.x);
}

// FDK takes caller frames only where they follow the nominal orbit: every
// x, y, z of src, detS, detU, detV and angle within 1e-3 of the views the
// scan builds (src/interface/YkReconstructionApi.cpp:156-167)
bool near_nominal(const SConeProjGeomVec& f, const ykb_cone_view& v)
{
    const float4 a[] = {f.src, f.detS, f.detU, f.detV, f.angle};
    const ykb_float4 b[] = {v.src, v.detS, v.detU, v.detV, v.angle};
    for (int j = 0; j < 5; ++j)
        if (std::abs(a[j].x - b[j].x) > 1e-3f || std::abs(a[j].y - b[j].y) > 1e-3f ||
            std::abs(a[j].z - b[j].z) > 1e-3f)
            return false;
    return true;
}

// SRigidTransform::aroundEulerPoint(centre, rx, ry, rz).inverse() applied to
// a view (include/YKCBCT/geometry/YkRigidTransform.hpp,
// transformProjectionGeometry in YkProjectionGeometry.hpp:229-247)
void pose_views(std::vector<ykb_cone_view>& views, const SForwardProjectionPose& pose,
    const float3& centre)
{
    const double cx = std::cos(pose.rotation_x_rad), sx = std::sin(pose.rotation_x_rad);
    const double cy = std::cos(pose.rotation_y_rad), sy = std::sin(pose.rotation_y_rad);
    const double cz = std::cos(pose.rotation_z_rad), sz = std::sin(pose.rotation_z_rad);
    // R = Rz Ry Rx; the inverse rotation is R^T about the same centre
    const double R[3][3] = {
        {cz * cy, cz * sy * sx - sz * cx, cz * sy * cx + sz * sx},
        {sz * cy, sz * sy * sx + cz * cx, sz * sy * cx - cz * sx},
        {-sy, cy * sx, cy * cx}};
    auto inv_vec = [&](const ykb_float4& v) {
        ykb_float4 r = v;
        r.x = static_cast<float>(R[0][0] * v.x + R[1][0] * v.y + R[2][0] * v.z);
        r.y = static_cast<float>(R[0][1] * v.x + R[1][1] * v.y + R[2][1] * v.z);
        r.z = static_cast<float>(R[0][2] * v.x + R[1][2] * v.y + R[2][2] * v.z);
        return r;
    };
    auto inv_pt = [&](const ykb_float4& p) {
        ykb_float4 d = p;
        d.x = p.x - centre.x; d.y = p.y - centre.y; d.z = p.z - centre.z;
        ykb_float4 r = inv_vec(d);
        r.x += centre.x; r.y += centre.y; r.z += centre.z;
        return r;
    };
    for (auto& v : views) {
        v.src = inv_pt(v.src);
        v.detS = inv_pt(v.detS);
        v.detU = inv_vec(v.detU);
        v.detV = inv_vec(v.detV);
    }
}

struct DeviceScratch {
    void* ptr = nullptr;
    size_t bytes = 0;
    bool ensure(size_t n)
    {
        if (bytes >= n) return true;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        if (cudaMalloc(&ptr, n) != cudaSuccess) { cudaGetLastError(); return false; }
        bytes = n;
        return true;
    }
    void reset()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

class Session final : public IReconstructionSession {
public:
    ~Session() override { release(); }

    bool initialize(const SSystemSpec& system) override
    {
        release();
        clear_();
        if (!has_bytes(system.struct_size, offsetof(SSystemSpec, device) + sizeof(system.device)))
            return fail_(EApiErrorCode::InvalidConfig, "SSystemSpec struct_size is too small (truncated)");
        if (system.api_version != 2)
            return fail_(EApiErrorCode::InvalidConfig, "unsupported SSystemSpec api_version");
        const auto& g = system.geometry;
        const auto& r = system.reconstruction;
        // caller frames: the tail counts only when struct_size covers it whole
        // (src/interface/YkReconstructionApi.cpp:144-168)
        const bool frame_tail = has_bytes(system.struct_size,
            offsetof(SSystemSpec, flat_frame_count) + sizeof(system.flat_frame_count));
        if (system.struct_size > offsetof(SSystemSpec, flat_frames) && !frame_tail)
            return fail_(EApiErrorCode::InvalidConfig, "Truncated flat-frame tail");
        const SConeProjGeomVec* frames = frame_tail ? system.flat_frames : nullptr;
        const int frame_count = frame_tail ? system.flat_frame_count : 0;
        if ((frames == nullptr) != (frame_count == 0) || frame_count < 0)
            return fail_(EApiErrorCode::InvalidConfig, "Invalid flat-frame buffer/count");
        if (frames) {
            const auto p = r.pipeline;
            if (g.detector != EDetectorKind::Flat ||
                (g.trajectory != ETrajectoryKind::Circular && g.trajectory != ETrajectoryKind::Helical) ||
                (p != EPipeline::ForwardProjection && p != EPipeline::SART && p != EPipeline::SIRT &&
                 p != EPipeline::OSSART && p != EPipeline::CGLS && p != EPipeline::FDK &&
                 p != EPipeline::WFBP))
                return fail_(EApiErrorCode::UnsupportedCombination,
                    "Unsupported external flat-frame algorithm");
        }
        if (static_cast<int>(g.detector) < 0 || static_cast<int>(g.detector) > 1 ||
            static_cast<int>(g.trajectory) < 0 || static_cast<int>(g.trajectory) > 3 ||
            static_cast<int>(r.pipeline) < 0 || static_cast<int>(r.pipeline) > 11)
            return fail_(EApiErrorCode::InvalidConfig, "invalid pipeline, detector or trajectory enum");
        if (g.detector != EDetectorKind::Flat || g.trajectory != ETrajectoryKind::Circular)
            return fail_(EApiErrorCode::UnsupportedCombination,
                "this library implements the flat-panel circular trajectory only");
        if (r.pipeline != EPipeline::FDK && r.pipeline != EPipeline::ForwardProjection)
            return fail_(EApiErrorCode::UnsupportedCombination,
                "this library implements the FDK and ForwardProjection pipelines only");
        if (static_cast<int>(r.forward_projector) < 0 || static_cast<int>(r.forward_projector) > 3 ||
            static_cast<int>(r.back_projector) < 0 || static_cast<int>(r.back_projector) > 5)
            return fail_(EApiErrorCode::InvalidConfig, "invalid forward/back projector selection");
        const auto& pose = g.forward_projection_pose;
        if (!std::isfinite(pose.rotation_x_rad) || !std::isfinite(pose.rotation_y_rad) ||
            !std::isfinite(pose.rotation_z_rad))
            return fail_(EApiErrorCode::InvalidGeometry,
                "Forward-projection volume rotation must contain finite radians");
        // the reference's regularisation and statistical tails: truncation is
        // an error; a regularisation plugin belongs to its algebraic solvers
        // (src/interface/YkReconstructionApi.cpp:207-222,241-244)
        if (system.struct_size > offsetof(SSystemSpec, regularization) &&
            !has_bytes(system.struct_size,
                offsetof(SSystemSpec, regularization) + sizeof(system.regularization)))
            return fail_(EApiErrorCode::InvalidConfig, "SSystemSpec regularization tail is truncated");
        if (has_bytes(system.struct_size,
                offsetof(SSystemSpec, regularization) + sizeof(system.regularization)) &&
            system.regularization.plugin_id && system.regularization.plugin_id[0] &&
            std::string(system.regularization.plugin_id) != "none")
            return fail_(EApiErrorCode::UnsupportedCombination,
                "TV plugins currently support flat SART/SIRT/OSSART only");
        if (system.struct_size > offsetof(SSystemSpec, statistical) &&
            !has_bytes(system.struct_size,
                offsetof(SSystemSpec, statistical) + sizeof(system.statistical)))
            return fail_(EApiErrorCode::InvalidConfig, "SSystemSpec statistical tail is truncated");
        if (r.pipeline == EPipeline::ForwardProjection &&
            r.forward_projector == EForwardProjector::SeparableFootprint)
            return fail_(EApiErrorCode::UnsupportedCombination,
                "forward projection here is Joseph or Siddon (EForwardProjector::SeparableFootprint "
                "is not implemented)");
        // resolveForwardProjector maps Automatic to Siddon for flat detectors
        // (src/interface/YkProjectorSelection.hpp:11-24)
        fp_task_ = r.forward_projector == EForwardProjector::Joseph ? YKB_TASK_FP_JOSEPH
                                                                    : YKB_TASK_FP_SIDDON;
        if (g.volume.nx <= 0 || g.volume.ny <= 0 || g.volume.nz <= 0 ||
            !(g.volume.voxel_x_mm > 0.f) || !(g.volume.voxel_y_mm > 0.f) ||
            !(g.volume.voxel_z_mm > 0.f) || !std::isfinite(g.volume.center_mm.x) ||
            !std::isfinite(g.volume.center_mm.y) || !std::isfinite(g.volume.center_mm.z))
            return fail_(EApiErrorCode::InvalidGeometry, "invalid volume grid");

        ykb_circular_flat spec{};
        spec.total_views = g.circular.total_views;
        spec.views_per_turn = g.circular.views_per_turn;
        spec.start_angle_rad = g.circular.start_angle_rad;
        spec.rotation_direction = g.circular.rotation_direction;
        spec.sid_mm = g.circular.sid_mm;
        spec.sdd_mm = g.circular.sdd_mm;
        spec.z_mm = g.circular.z_mm;
        spec.source_offset_mm[0] = g.circular.source_offset_mm.x;
        spec.source_offset_mm[1] = g.circular.source_offset_mm.y;
        spec.source_offset_mm[2] = g.circular.source_offset_mm.z;
        spec.channels = g.flat_detector.channels;
        spec.rows = g.flat_detector.rows;
        spec.channel_size_mm = g.flat_detector.channel_size_mm;
        spec.row_size_mm = g.flat_detector.row_size_mm;
        spec.offset_unv_mm[0] = g.flat_detector.pose.offset_unv_mm.x;
        spec.offset_unv_mm[1] = g.flat_detector.pose.offset_unv_mm.y;
        spec.offset_unv_mm[2] = g.flat_detector.pose.offset_unv_mm.z;
        spec.tilt_u_rad = g.flat_detector.pose.tilt_u_rad;
        spec.tilt_v_rad = g.flat_detector.pose.tilt_v_rad;
        spec.tilt_n_rad = g.flat_detector.pose.tilt_n_rad;
        if (spec.total_views <= 0)
            return fail_(EApiErrorCode::InvalidGeometry, "total_views must be positive");
        views_.assign(static_cast<size_t>(spec.total_views), ykb_cone_view{});
        // caller frames replace the built views: FDK only near the nominal
        // orbit (so the orbit is built to compare), forward projection any
        // valid frames (the reference then builds no orbit,
        // src/common/YkExecutionContext.hpp:23-38)
        const bool frames_only = frames && r.pipeline == EPipeline::ForwardProjection;
        if (!frames_only && ykb_build_circular_flat(&spec, views_.data(), spec.total_views) != YKB_OK) {
            views_.clear();
            return fail_(EApiErrorCode::InvalidGeometry, ykb_last_error());
        }
        float parker_start = spec.start_angle_rad;
        int parker_direction = spec.rotation_direction;
        if (frames) {
            if (frame_count != spec.total_views) {
                views_.clear();
                return fail_(EApiErrorCode::InvalidGeometry,
                    r.pipeline == EPipeline::FDK
                        ? "Analytic external geometry requires matching nominal trajectory"
                        : "flat_frame_count must equal the scan's total_views");
            }
            for (int i = 0; i < frame_count; ++i) {
                if (r.pipeline == EPipeline::FDK && !near_nominal(frames[i], views_[i])) {
                    views_.clear();
                    return fail_(EApiErrorCode::UnsupportedCombination,
                        "External frames do not match analytic trajectory assumptions; use "
                        "iterative reconstruction");
                }
                if (!valid_frame(frames[i])) {
                    views_.clear();
                    return fail_(EApiErrorCode::InvalidGeometry,
                        "external frames must be finite with orthogonal detU and detV");
                }
            }
            for (int i = 0; i < frame_count; ++i) views_[i] = to_view(frames[i]);
            // the frames' angles are the only angle source: Parker starts at
            // the first and turns the way the first two go
            // (src/interface/YkSession.cpp:131-139)
            parker_start = frames[0].angle.x;
            if (frame_count >= 2) parker_direction = frames[1].angle.x >= frames[0].angle.x ? 1 : -1;
        }

        volume_ = ykb_volume{g.volume.nx, g.volume.ny, g.volume.nz, g.volume.voxel_x_mm,
            g.volume.voxel_y_mm, g.volume.voxel_z_mm, g.volume.center_mm.x, g.volume.center_mm.y,
            g.volume.center_mm.z};
        nu_ = spec.channels;
        nv_ = spec.rows;
        device_ = system.device;
        pipeline_ = r.pipeline;
        int count = 0;
        if (device_ < 0 || cudaGetDeviceCount(&count) != cudaSuccess || device_ >= count) {
            cudaGetLastError();
            return fail_(EApiErrorCode::InvalidGeometry, "invalid GPU selection");
        }
        ykb::DeviceGuard guard(device_);
        if (pipeline_ == EPipeline::FDK) {
            const auto& f = r.fdk.filter;
            if (static_cast<int>(f.type) < 0 || static_cast<int>(f.type) > 9 ||
                !std::isfinite(f.cutoff) || !(f.cutoff > 0.f) || f.cutoff > .5f ||
                !std::isfinite(f.gain) || !(f.gain > 0.f) || !std::isfinite(f.butterworth_order) ||
                !(f.butterworth_order > 0.f) || !std::isfinite(f.kaiser_beta) || f.kaiser_beta < 0.f ||
                !std::isfinite(f.tukey_alpha) || f.tukey_alpha < 0.f || f.tukey_alpha > 1.f) {
                views_.clear();
                return fail_(EApiErrorCode::InvalidGeometry, "invalid analytic filter parameters");
            }
            const ykb_filter filt{static_cast<int>(f.type), f.cutoff, f.gain, f.butterworth_order,
                f.kaiser_beta, f.tukey_alpha};
            const float range = ykb_regular_scan_range(spec.total_views, spec.views_per_turn);
            // Parker: EParkerMode values map one to one; Auto weights short
            // scans (resolveParkerEnabled, YkSystemReconstruction.hpp:29-39)
            if (ykb_fdk_plan_create_ex(views_.data(), spec.total_views, nu_, nv_, range,
                    parker_start, parker_direction, &volume_, &filt,
                    YKB_PRECISION_FP32, static_cast<int>(r.fdk.parker.mode), device_,
                    &fdk_) != YKB_OK) {
                const std::string msg = ykb_last_error();
                release();
                return fail_(EApiErrorCode::InvalidGeometry, msg.c_str());
            }
        } else {
            if (pose.enabled) pose_views(views_, pose, g.volume.center_mm);
            if (ykb_joseph_plan_create(views_.data(), spec.total_views, nu_, nv_, &volume_, device_,
                    &joseph_) != YKB_OK) {
                const std::string msg = ykb_last_error();
                release();
                return fail_(EApiErrorCode::InvalidGeometry, msg.c_str());
            }
        }
        if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            release();
            return fail_(EApiErrorCode::CudaError, "cudaStreamCreate failed");
        }
        view_count_ = spec.total_views;
        received_ = 0;
        initialized_ = true;
        return true;
    }

    bool execute(const SExecutionRequest& request) override
    {
        clear_();
        if (!initialized_)
            return fail_(EApiErrorCode::StreamingStateError, "the session is not initialized");
        if (!has_bytes(request.struct_size,
                offsetof(SExecutionRequest, iteration_count) + sizeof(request.iteration_count)))
            return fail_(EApiErrorCode::InvalidConfig, "SExecutionRequest struct_size is too small (truncated)");
        if (request.struct_size > offsetof(SExecutionRequest, progress_callback) &&
            request.struct_size < offsetof(SExecutionRequest, progress_user_data) +
                sizeof(request.progress_user_data))
            return fail_(EApiErrorCode::InvalidConfig, "SExecutionRequest progress tail is truncated");
        if (request.api_version != 2)
            return fail_(EApiErrorCode::InvalidConfig, "unsupported SExecutionRequest api_version");
        // projection readers and statistical weights feed the reference's
        // iterative pipelines only (src/interface/YkReconstructionApi.cpp:327-343)
        if (request.struct_size > offsetof(SExecutionRequest, projection_read) &&
            request.struct_size < offsetof(SExecutionRequest, projection_batch_mib) +
                sizeof(request.projection_batch_mib))
            return fail_(EApiErrorCode::InvalidConfig, "SExecutionRequest projection source tail is truncated");
        const bool weights_tail = has_bytes(request.struct_size,
            offsetof(SExecutionRequest, projection_weights_read_user_data) +
                sizeof(request.projection_weights_read_user_data));
        if (request.struct_size > offsetof(SExecutionRequest, projection_weights) && !weights_tail)
            return fail_(EApiErrorCode::InvalidConfig, "SExecutionRequest statistical weights tail is truncated");
        if (weights_tail && (request.projection_weights.data || request.projection_weights_read))
            return fail_(EApiErrorCode::UnsupportedCombination,
                "Projection W is only accepted when statistical diagonal weights are enabled");
        const bool source_tail = has_bytes(request.struct_size,
            offsetof(SExecutionRequest, projection_batch_mib) + sizeof(request.projection_batch_mib));
        if (source_tail && request.projection_read)
            return fail_(EApiErrorCode::UnsupportedCombination,
                "Projection reader requires supported flat SART/SIRT/OSSART or TIGRE "
                "SART/OS-SART/SIRT/TV without Nesterov/FDK initialization");
        if (!request.projection.data || !request.volume.data ||
            !valid_location(request.projection.location) || !valid_location(request.volume.location))
            return fail_(EApiErrorCode::InvalidBuffer, "null projection/volume buffer or invalid location");
        const int offset = request.view_offset;
        const int count = request.view_count > 0 ? request.view_count : view_count_;
        if (offset < 0 || count <= 0 || offset > view_count_ - count)
            return fail_(EApiErrorCode::InvalidConfig, "view_offset/view_count outside the prepared views");
        const bool fdk = pipeline_ == EPipeline::FDK;
        if (fdk) {
            if (offset != received_)
                return fail_(EApiErrorCode::StreamingStateError,
                    "FDK batches must be submitted with contiguous view_offset (no gaps or repeats)");
            if (received_ > 0 && request.clear_output)
                return fail_(EApiErrorCode::StreamingStateError,
                    "only the first FDK batch may set clear_output");
        } else if (offset != 0 || count != view_count_) {
            return fail_(EApiErrorCode::StreamingStateError,
                "this pipeline takes the complete view sequence from view_offset 0");
        }
        const size_t view_elems = static_cast<size_t>(nu_) * nv_;
        const size_t vol_elems = static_cast<size_t>(volume_.nx) * volume_.ny * volume_.nz;
        if (request.projection.element_count < view_elems * count ||
            request.volume.element_count < vol_elems)
            return fail_(EApiErrorCode::InvalidBuffer,
                "projection/volume element_count smaller than this execution needs");
        ykb::DeviceGuard guard(device_);
        const bool ok = fdk ? run_fdk_(request, offset, count) : run_fp_(request, count);
        if (!ok) return false;
        if (fdk) received_ += count;
        return true;
    }

    bool isInitialized() const override { return initialized_; }
    EApiErrorCode lastError() const override { return code_; }
    const char* lastErrorMessage() const override { return message_.c_str(); }

    void reset() override { received_ = 0; }

    void release() override
    {
        if (stream_) cudaStreamSynchronize(stream_);
        if (fdk_) ykb_fdk_plan_destroy(fdk_);
        if (joseph_) ykb_joseph_plan_destroy(joseph_);
        fdk_ = nullptr;
        joseph_ = nullptr;
        proj_scratch_.reset();
        vol_scratch_.reset();
        if (stream_) cudaStreamDestroy(stream_);
        stream_ = nullptr;
        views_.clear();
        view_count_ = received_ = 0;
        initialized_ = false;
    }

private:
    bool cuda_fail_(cudaError_t e, const char* what)
    {
        cudaGetLastError();
        return fail_(EApiErrorCode::CudaError,
            (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
    }

    bool run_fdk_(const SExecutionRequest& r, int offset, int count)
    {
        const size_t vol_bytes = static_cast<size_t>(volume_.nx) * volume_.ny * volume_.nz * sizeof(float);
        float* d_vol = r.volume.data;
        if (r.volume.location == EMemoryLocation::Host) {
            // a host volume accumulates in device scratch across batches and is
            // copied back once the last batch has arrived
            if (!vol_scratch_.ensure(vol_bytes))
                return fail_(EApiErrorCode::CudaError, "device volume scratch allocation failed");
            d_vol = static_cast<float*>(vol_scratch_.ptr);
        }
        // host projections stream in batches, their copies overlapping the
        // kernels of earlier batches (the reference copies each 32-view chunk
        // synchronously: YkFdkPipeline.hpp:454-457)
        const bool last = received_ + count == view_count_;
        const bool host_vol = r.volume.location == EMemoryLocation::Host;
        ykb_status st;
        if (r.projection.location == EMemoryLocation::Host && host_vol && last)
            // the final batch also returns the volume, its download
            // overlapping the last backprojection slab by slab
            st = ykb_fdk_execute_host_out(fdk_, r.projection.data, YKB_DTYPE_F32, offset, count,
                d_vol, r.volume.data, r.clear_output ? 1 : 0, stream_);
        else if (r.projection.location == EMemoryLocation::Host)
            st = ykb_fdk_execute_host(fdk_, r.projection.data, YKB_DTYPE_F32, offset, count, d_vol,
                r.clear_output ? 1 : 0, stream_);
        else
            st = ykb_fdk_execute(fdk_, r.projection.data, YKB_DTYPE_F32, offset, count, d_vol,
                r.clear_output ? 1 : 0, stream_);
        if (st != YKB_OK) return fail_(EApiErrorCode::CudaError, ykb_last_error());
        if (host_vol && last && r.projection.location != EMemoryLocation::Host) {
            const cudaError_t e = cudaMemcpyAsync(r.volume.data, d_vol, vol_bytes,
                cudaMemcpyDeviceToHost, stream_);
            if (e != cudaSuccess) return cuda_fail_(e, "volume download");
        }
        if (ykb_fdk_check(fdk_, stream_) != YKB_OK)
            return fail_(EApiErrorCode::CudaError, ykb_last_error());
        return true;
    }

    bool run_fp_(const SExecutionRequest& r, int count)
    {
        const size_t proj_bytes = static_cast<size_t>(nu_) * nv_ * count * sizeof(float);
        const size_t vol_bytes = static_cast<size_t>(volume_.nx) * volume_.ny * volume_.nz * sizeof(float);
        const float* d_vol = r.volume.data;
        if (r.volume.location == EMemoryLocation::Host) {
            if (!vol_scratch_.ensure(vol_bytes))
                return fail_(EApiErrorCode::CudaError, "device volume scratch allocation failed");
            const cudaError_t e = cudaMemcpyAsync(vol_scratch_.ptr, r.volume.data, vol_bytes,
                cudaMemcpyHostToDevice, stream_);
            if (e != cudaSuccess) return cuda_fail_(e, "volume upload");
            d_vol = static_cast<const float*>(vol_scratch_.ptr);
        }
        float* d_proj = r.projection.data;
        if (r.projection.location == EMemoryLocation::Host) {
            if (!proj_scratch_.ensure(proj_bytes))
                return fail_(EApiErrorCode::CudaError, "device projection scratch allocation failed");
            d_proj = static_cast<float*>(proj_scratch_.ptr);
        }
        if (ykb_operator_apply(joseph_, fp_task_, d_vol, d_proj, 0, stream_) != YKB_OK)
            return fail_(EApiErrorCode::CudaError, ykb_last_error());
        if (r.projection.location == EMemoryLocation::Host) {
            const cudaError_t e = cudaMemcpyAsync(r.projection.data, d_proj, proj_bytes,
                cudaMemcpyDeviceToHost, stream_);
            if (e != cudaSuccess) return cuda_fail_(e, "projection download");
        }
        const cudaError_t e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) return cuda_fail_(e, "forward projection");
        return true;
    }

    bool fail_(EApiErrorCode code, const char* message)
    {
        code_ = code;
        message_ = message ? message : "";
        return false;
    }
    void clear_()
    {
        code_ = EApiErrorCode::None;
        message_.clear();
    }

    std::vector<ykb_cone_view> views_;
    ykb_volume volume_{};
    int nu_ = 0, nv_ = 0, device_ = 0;
    EPipeline pipeline_ = EPipeline::FDK;
    int view_count_ = 0, received_ = 0;
    bool initialized_ = false;
    ykb_fdk_plan* fdk_ = nullptr;
    ykb_joseph_plan* joseph_ = nullptr;
    int fp_task_ = YKB_TASK_FP_JOSEPH;  // FP_Joseph or FP_Siddon
    cudaStream_t stream_ = nullptr;
    DeviceScratch proj_scratch_, vol_scratch_;
    EApiErrorCode code_ = EApiErrorCode::None;
    std::string message_;
};

} // namespace

IReconstructionSession* ReconstructionSessionFactory::create()
{
    return new (std::nothrow) Session();
}

void ReconstructionSessionFactory::destroy(IReconstructionSession* session) { delete session; }

} // namespace YK
