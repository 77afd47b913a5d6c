// One client source compiled twice, against the reference's public API header
// (include/YKCBCT/interface/YkReconstructionApi.hpp, -DYKB_LAYOUT_REFERENCE)
// and against libykb's include/ykb_session.hpp.  It sets the members a caller
// of the reference sets, then prints every public struct's size, each
// member's offset and the default value of each scalar member, one per line.
// tests/test_session.py runs both builds and requires identical output: the
// same source compiles unchanged and the binary layouts agree.
#ifdef YKB_LAYOUT_REFERENCE
#include "YKCBCT/interface/YkReconstructionApi.hpp"
#else
#include "ykb_session.hpp"
#endif

#include <cstddef>
#include <cstdio>
#include <type_traits>

using namespace YK;

namespace {

template <typename T>
double as_number(const T& v)
{
    if constexpr (std::is_enum_v<T>) return static_cast<double>(static_cast<long long>(v));
    else if constexpr (std::is_pointer_v<T>) return v ? 1.0 : 0.0;
    else return static_cast<double>(v);
}

#define SIZE(T) std::printf("sizeof %s %zu\n", #T, sizeof(T))
#define MEMBER(T, m) std::printf("offsetof %s.%s %zu\n", #T, #m, offsetof(T, m))
#define SCALAR(T, m) do { MEMBER(T, m); std::printf("default %s.%s %.9g\n", #T, #m, as_number(T{}.m)); } while (0)

// a client of the session: the members its callers fill in
SSystemSpec client_spec(const SConeProjGeomVec* frames, int count)
{
    SSystemSpec s{};
    s.geometry.detector = EDetectorKind::Flat;
    s.geometry.trajectory = ETrajectoryKind::Circular;
    s.geometry.circular.total_views = count;
    s.geometry.circular.views_per_turn = count;
    s.geometry.circular.sid_mm = 500.f;
    s.geometry.circular.sdd_mm = 1000.f;
    s.geometry.helical.pitch_mm_per_turn = 0.f;
    s.geometry.flat_detector.channels = 192;
    s.geometry.flat_detector.rows = 128;
    s.geometry.flat_detector.channel_size_mm = 0.8f;
    s.geometry.flat_detector.row_size_mm = 0.8f;
    s.geometry.cylindrical_detector.curvature_radius_mm = 0.f;
    s.geometry.volume = {128, 128, 128, 0.5f, 0.5f, 0.5f, {0.f, 0.f, 0.f}};
    s.reconstruction.pipeline = EPipeline::FDK;
    s.reconstruction.forward_projector = EForwardProjector::Joseph;
    s.reconstruction.fdk.parker.mode = EParkerMode::Auto;
    s.reconstruction.fdk.filter.type = EFdkFilter::SheppLogan;
    s.reconstruction.iterative.iterations = 10;
    s.reconstruction.cgls.robust_restart = true;
    s.regularization.plugin_id = nullptr;
    s.statistical.optimizer.iterations = 10;
    s.flat_frames = frames;
    s.flat_frame_count = frames ? count : 0;
    return s;
}

} // namespace

int main()
{
    const SSystemSpec spec = client_spec(nullptr, 180);
    SExecutionRequest req{};
    req.projection = {nullptr, EMemoryLocation::Host, 0};
    req.volume = {nullptr, EMemoryLocation::Device, 0};
    req.view_offset = 0;
    req.view_count = 0;
    std::printf("client %u %u %d\n", spec.struct_size, req.struct_size,
        spec.geometry.circular.total_views);

    SIZE(SConeProjGeomVec);
    MEMBER(SConeProjGeomVec, src); MEMBER(SConeProjGeomVec, detS); MEMBER(SConeProjGeomVec, detU);
    MEMBER(SConeProjGeomVec, detV); MEMBER(SConeProjGeomVec, angle);
    SIZE(SDetectorPoseSpec);
    MEMBER(SDetectorPoseSpec, offset_unv_mm); SCALAR(SDetectorPoseSpec, tilt_u_rad);
    SCALAR(SDetectorPoseSpec, tilt_v_rad); SCALAR(SDetectorPoseSpec, tilt_n_rad);
    SIZE(SRegularCircularScanSpec);
    SCALAR(SRegularCircularScanSpec, total_views); SCALAR(SRegularCircularScanSpec, views_per_turn);
    SCALAR(SRegularCircularScanSpec, start_angle_rad); SCALAR(SRegularCircularScanSpec, rotation_direction);
    SCALAR(SRegularCircularScanSpec, sid_mm); SCALAR(SRegularCircularScanSpec, sdd_mm);
    SCALAR(SRegularCircularScanSpec, z_mm); MEMBER(SRegularCircularScanSpec, source_offset_mm);
    SIZE(SRegularHelicalScanSpec);
    SCALAR(SRegularHelicalScanSpec, total_views); SCALAR(SRegularHelicalScanSpec, views_per_turn);
    SCALAR(SRegularHelicalScanSpec, start_angle_rad); SCALAR(SRegularHelicalScanSpec, rotation_direction);
    SCALAR(SRegularHelicalScanSpec, sid_mm); SCALAR(SRegularHelicalScanSpec, sdd_mm);
    SCALAR(SRegularHelicalScanSpec, start_z_mm); SCALAR(SRegularHelicalScanSpec, pitch_mm_per_turn);
    MEMBER(SRegularHelicalScanSpec, source_offset_mm);
    SIZE(SFlatDetectorSpec);
    SCALAR(SFlatDetectorSpec, channels); SCALAR(SFlatDetectorSpec, rows);
    SCALAR(SFlatDetectorSpec, channel_size_mm); SCALAR(SFlatDetectorSpec, row_size_mm);
    MEMBER(SFlatDetectorSpec, pose);
    SIZE(SCylDetectorSpec);
    SCALAR(SCylDetectorSpec, channels); SCALAR(SCylDetectorSpec, rows);
    SCALAR(SCylDetectorSpec, channel_arc_mm); SCALAR(SCylDetectorSpec, row_size_mm);
    SCALAR(SCylDetectorSpec, curvature_radius_mm); MEMBER(SCylDetectorSpec, pose);
    SIZE(SVolumeGridSpec);
    SCALAR(SVolumeGridSpec, nx); SCALAR(SVolumeGridSpec, ny); SCALAR(SVolumeGridSpec, nz);
    SCALAR(SVolumeGridSpec, voxel_x_mm); SCALAR(SVolumeGridSpec, voxel_y_mm);
    SCALAR(SVolumeGridSpec, voxel_z_mm); MEMBER(SVolumeGridSpec, center_mm);
    SIZE(SForwardProjectionPose);
    SCALAR(SForwardProjectionPose, enabled); SCALAR(SForwardProjectionPose, rotation_x_rad);
    SCALAR(SForwardProjectionPose, rotation_y_rad); SCALAR(SForwardProjectionPose, rotation_z_rad);
    SIZE(SSystemConfig);
    SCALAR(SSystemConfig, detector); SCALAR(SSystemConfig, trajectory);
    MEMBER(SSystemConfig, circular); MEMBER(SSystemConfig, helical);
    MEMBER(SSystemConfig, flat_detector); MEMBER(SSystemConfig, cylindrical_detector);
    MEMBER(SSystemConfig, volume); MEMBER(SSystemConfig, forward_projection_pose);
    SIZE(SPlanarSourceOrbitSpec);
    SCALAR(SPlanarSourceOrbitSpec, total_views); SCALAR(SPlanarSourceOrbitSpec, start_angle_rad);
    SCALAR(SPlanarSourceOrbitSpec, scan_range_rad); SCALAR(SPlanarSourceOrbitSpec, rotation_direction);
    SCALAR(SPlanarSourceOrbitSpec, sid_mm); SCALAR(SPlanarSourceOrbitSpec, detector_y_mm);
    SCALAR(SPlanarSourceOrbitSpec, source_orbit_radius_mm);
    SCALAR(SPlanarSourceOrbitSpec, source_lateral_offset_mm);
    SCALAR(SPlanarSourceOrbitSpec, reconstruction_channels);
    SCALAR(SPlanarSourceOrbitSpec, reconstruction_rows); SCALAR(SPlanarSourceOrbitSpec, resample_mode);
    SIZE(SNikonTiltedCtSpec);
    SCALAR(SNikonTiltedCtSpec, total_views); SCALAR(SNikonTiltedCtSpec, start_angle_rad);
    SCALAR(SNikonTiltedCtSpec, scan_range_rad); SCALAR(SNikonTiltedCtSpec, rotation_direction);
    SCALAR(SNikonTiltedCtSpec, sid_mm); SCALAR(SNikonTiltedCtSpec, sdd_mm);
    SCALAR(SNikonTiltedCtSpec, tilt_rad); SCALAR(SNikonTiltedCtSpec, tilt_axis_azimuth_rad);
    MEMBER(SNikonTiltedCtSpec, source_offset_mm); MEMBER(SNikonTiltedCtSpec, rotation_axis_pivot_mm);
    SIZE(SNonStandardGeometrySpec);
    MEMBER(SNonStandardGeometrySpec, planar_source_orbit); MEMBER(SNonStandardGeometrySpec, nikon_tilted);
    SIZE(SAnalyticFilterParams);
    SCALAR(SAnalyticFilterParams, type); SCALAR(SAnalyticFilterParams, cutoff);
    SCALAR(SAnalyticFilterParams, gain); SCALAR(SAnalyticFilterParams, butterworth_order);
    SCALAR(SAnalyticFilterParams, kaiser_beta); SCALAR(SAnalyticFilterParams, tukey_alpha);
    SIZE(SParkerScanSpec); SCALAR(SParkerScanSpec, mode);
    SIZE(SFdkAlgoParams); MEMBER(SFdkAlgoParams, parker); MEMBER(SFdkAlgoParams, filter);
    SIZE(SIterAlgoParams);
    SCALAR(SIterAlgoParams, iterations); SCALAR(SIterAlgoParams, relaxation); SCALAR(SIterAlgoParams, subsets);
    SIZE(SCglsAlgoParams);
    SCALAR(SCglsAlgoParams, minimum_iterations); SCALAR(SCglsAlgoParams, check_interval);
    SCALAR(SCglsAlgoParams, patience); SCALAR(SCglsAlgoParams, relative_residual);
    SCALAR(SCglsAlgoParams, robust_restart);
    SIZE(SPwlsAlgoParams);
    SCALAR(SPwlsAlgoParams, regularizer); SCALAR(SPwlsAlgoParams, regularization);
    SCALAR(SPwlsAlgoParams, huber_delta); SCALAR(SPwlsAlgoParams, epsilon);
    SCALAR(SPwlsAlgoParams, lower_bound); SCALAR(SPwlsAlgoParams, upper_bound);
    SCALAR(SPwlsAlgoParams, use_projection_weights);
    SIZE(STigreGradientAlgoParams);
    SCALAR(STigreGradientAlgoParams, method); SCALAR(STigreGradientAlgoParams, block_size);
    SCALAR(STigreGradientAlgoParams, lambda_reduction); SCALAR(STigreGradientAlgoParams, nesterov_relaxation);
    SCALAR(STigreGradientAlgoParams, fdk_initialization); SCALAR(STigreGradientAlgoParams, non_negative);
    SCALAR(STigreGradientAlgoParams, tv_iterations); SCALAR(STigreGradientAlgoParams, tv_alpha);
    SCALAR(STigreGradientAlgoParams, tv_alpha_reduction);
    SCALAR(STigreGradientAlgoParams, maximum_update_ratio); SCALAR(STigreGradientAlgoParams, max_l2_error);
    SIZE(SWfbpAlgoParams); SCALAR(SWfbpAlgoParams, redundancy_flat); MEMBER(SWfbpAlgoParams, filter);
    SIZE(SReconstructionSpec);
    SCALAR(SReconstructionSpec, pipeline); SCALAR(SReconstructionSpec, forward_projector);
    SCALAR(SReconstructionSpec, back_projector); MEMBER(SReconstructionSpec, fdk);
    MEMBER(SReconstructionSpec, iterative); MEMBER(SReconstructionSpec, cgls);
    MEMBER(SReconstructionSpec, pwls); MEMBER(SReconstructionSpec, tigre); MEMBER(SReconstructionSpec, wfbp);
    SIZE(SAlgebraicRegularizationSpec);
    SCALAR(SAlgebraicRegularizationSpec, plugin_id); SCALAR(SAlgebraicRegularizationSpec, strength);
    SCALAR(SAlgebraicRegularizationSpec, huber_delta); SCALAR(SAlgebraicRegularizationSpec, step_size);
    SCALAR(SAlgebraicRegularizationSpec, inner_iterations); SCALAR(SAlgebraicRegularizationSpec, dimensions);
    SCALAR(SAlgebraicRegularizationSpec, epsilon);
    SCALAR(SAlgebraicRegularizationSpec, strength_reduction);
    SCALAR(SAlgebraicRegularizationSpec, non_negative);
    SIZE(SDataFidelitySpec);
    SCALAR(SDataFidelitySpec, kind); SCALAR(SDataFidelitySpec, use_projection_weights);
    SCALAR(SDataFidelitySpec, normalize_by_ray_count); SCALAR(SDataFidelitySpec, require_verified_adjoint);
    SCALAR(SDataFidelitySpec, scale);
    SIZE(SStatisticalRegularizationSpec);
    SCALAR(SStatisticalRegularizationSpec, plugin_id); SCALAR(SStatisticalRegularizationSpec, strength);
    SCALAR(SStatisticalRegularizationSpec, shape); SCALAR(SStatisticalRegularizationSpec, dimensions);
    SIZE(SStatisticalOptimizerSpec);
    SCALAR(SStatisticalOptimizerSpec, kind); SCALAR(SStatisticalOptimizerSpec, iterations);
    SCALAR(SStatisticalOptimizerSpec, step_size); SCALAR(SStatisticalOptimizerSpec, backtracking);
    SCALAR(SStatisticalOptimizerSpec, max_backtracking); SCALAR(SStatisticalOptimizerSpec, step_shrink);
    SCALAR(SStatisticalOptimizerSpec, relative_tolerance);
    SCALAR(SStatisticalOptimizerSpec, minimum_iterations);
    SIZE(SStatisticalConstraintSpec);
    SCALAR(SStatisticalConstraintSpec, lower_bound); SCALAR(SStatisticalConstraintSpec, upper_bound);
    SIZE(SStatisticalReconstructionSpec);
    MEMBER(SStatisticalReconstructionSpec, data_fidelity);
    MEMBER(SStatisticalReconstructionSpec, regularization);
    MEMBER(SStatisticalReconstructionSpec, optimizer);
    MEMBER(SStatisticalReconstructionSpec, constraints);
    SIZE(SSystemSpec);
    SCALAR(SSystemSpec, struct_size); SCALAR(SSystemSpec, api_version); MEMBER(SSystemSpec, geometry);
    MEMBER(SSystemSpec, reconstruction); SCALAR(SSystemSpec, device); MEMBER(SSystemSpec, nonstandard);
    MEMBER(SSystemSpec, regularization); MEMBER(SSystemSpec, statistical);
    SCALAR(SSystemSpec, flat_frames); SCALAR(SSystemSpec, flat_frame_count);
    SIZE(Buffer);
    SCALAR(Buffer, data); SCALAR(Buffer, location); SCALAR(Buffer, element_count);
    SIZE(SExecutionRequest);
    SCALAR(SExecutionRequest, struct_size); SCALAR(SExecutionRequest, api_version);
    MEMBER(SExecutionRequest, projection); MEMBER(SExecutionRequest, volume);
    SCALAR(SExecutionRequest, view_offset); SCALAR(SExecutionRequest, view_count);
    SCALAR(SExecutionRequest, clear_output); SCALAR(SExecutionRequest, iteration_count);
    SCALAR(SExecutionRequest, progress_callback); SCALAR(SExecutionRequest, progress_user_data);
    SCALAR(SExecutionRequest, projection_read); SCALAR(SExecutionRequest, projection_read_user_data);
    SCALAR(SExecutionRequest, projection_batch_views); SCALAR(SExecutionRequest, projection_batch_mib);
    MEMBER(SExecutionRequest, projection_weights); SCALAR(SExecutionRequest, projection_weights_read);
    SCALAR(SExecutionRequest, projection_weights_read_user_data);
    std::printf("enum %d %d %d %d %d %d\n", static_cast<int>(EPipeline::Statistical),
        static_cast<int>(EBackProjector::SeparableFootprint),
        static_cast<int>(EApiErrorCode::CudaError), static_cast<int>(ETrajectoryKind::NikonTilted),
        static_cast<int>(ETigreGradientMethodSpec::OsAwAsdPocs),
        static_cast<int>(EStatisticalOptimizer::RegularizedAlgebraic));
    return 0;
}
