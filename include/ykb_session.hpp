// ykb_session.hpp -- C++ Session layer of libykb for the flat-panel circular
// path: the types, members, member order, defaults and error behaviour of
// YKCBCT's public API (include/YKCBCT/interface/YkReconstructionApi.hpp:18-98
// and the headers it includes: YkReconstructionTypes.hpp,
// YkSystemReconstruction.hpp:9-19, geometry/YkGeometryBuilderTypes.hpp,
// geometry/YkSystemGeometry.hpp:24-32, geometry/YkNonStandardGeometrySpec.hpp,
// geometry/YkProjectionGeometry.hpp:12-18 and algorithms/*/Yk*Params.hpp), so
// that code written against that API compiles unchanged here and every public
// struct has the reference's size and member offsets
// (tests/session_layout.cpp compiles one client against both headers).
//
// Scope: flat detector, circular trajectory, EPipeline::FDK and
// EPipeline::ForwardProjection with EForwardProjector::Joseph, ::Siddon or
// ::Automatic (Siddon for a flat detector, as the reference resolves it),
// including caller geometry through SSystemSpec::flat_frames.  Members that
// only the reference's other algorithms read (helical and cylindrical specs,
// iterative / statistical / regularisation parameters, projection readers and
// weights) are declared with the reference's layout; initialize() and
// execute() reject requests that would need them with the reference's error
// codes (UnsupportedCombination for other pipelines, detectors and
// trajectories).
//
// This is a source-level interface over the C-ABI of ykb.h (the binary
// boundary); every execute() runs on the session's own CUDA stream and
// returns after the GPU work completes, as the reference's does.
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>

#include <vector_types.h>  // float3, float4, as the reference's public headers use

#if defined(_WIN32)
#define YKB_SESSION_API __declspec(dllexport)
#else
#define YKB_SESSION_API __attribute__((visibility("default")))
#endif

namespace YK {

// ---------------------------------------------------------------- enums ---
enum class EDetectorKind : int32_t { Flat, Cylindrical };
enum class ETrajectoryKind : int32_t { Circular, Helical, PlanarSourceOrbit, NikonTilted };

enum class EPipeline : int32_t {
    FDK, ForwardProjection, SIRT, OSSART, CGLS, PWLS, XFDK, CFDK, WFBP, TigreGradient, SART,
    Statistical,
};

enum class EMemoryLocation : int32_t { Host, Device };

enum class EForwardProjector : int32_t { Automatic, Siddon, Joseph, SeparableFootprint };
enum class EBackProjector : int32_t {
    Automatic, FdkPseudoMatched, SiddonRayDriven, Joseph, JosephV3, SeparableFootprint,
};

enum class EFdkFilter : int32_t {
    None = 0, RamLak = 1, SheppLogan = 2, Cosine = 3, Hann = 4, Hamming = 5, Blackman = 6,
    Butterworth = 7, Kaiser = 8, Tukey = 9,
};

enum class EParkerMode : int32_t { Auto, Disabled, Enabled };

enum class EPwlsRegularizerSpec : int32_t { None, Quadratic, Huber };

enum class ETigreGradientMethodSpec : int32_t {
    Sart, OsSart, Sirt, AsdPocs, OsAsdPocs, BAsdPocsBeta, Pcsd, OsPcsd, AwPcsd, OsAwPcsd,
    AwAsdPocs, OsAwAsdPocs,
};

enum class EPlanarResampleMode : int32_t { InPlaneRotated, PerspectiveOrthogonal };

enum class EStatisticalOptimizer : int32_t {
    GradientDescent = 0, Fista = 1, RegularizedAlgebraic = 2,
};
enum class EDataFidelityKind : int32_t { WeightedLeastSquares = 0 };

enum class EApiErrorCode : int32_t {
    None = 0, InvalidConfig, InvalidGeometry, UnsupportedCombination, AlgorithmUnderTest,
    InvalidBuffer, StreamingStateError, CudaError,
};

// ------------------------------------------------------------- geometry ---
// One view of a flat detector: source, centre of pixel (0,0), one-pixel
// steps along u and v, and the view angle in angle.x (80 bytes).
struct SConeProjGeomVec {
    float4 src;
    float4 detS;
    float4 detU;
    float4 detV;
    float4 angle;
};

// Detector pose in detector-local U, N, V (offset) and tilts about U, V, N.
struct SDetectorPoseSpec {
    float3 offset_unv_mm = {0.f, 0.f, 0.f};
    float tilt_u_rad = 0.f;
    float tilt_v_rad = 0.f;
    float tilt_n_rad = 0.f;
};

struct SRegularCircularScanSpec {
    int total_views = 0;
    int views_per_turn = 0;
    float start_angle_rad = 0.f;
    int rotation_direction = 1;
    float sid_mm = 0.f;
    float sdd_mm = 0.f;
    float z_mm = 0.f;
    float3 source_offset_mm = {0.f, 0.f, 0.f};
};

// Helical acquisition (declared for layout; rejected by this library).
struct SRegularHelicalScanSpec {
    int total_views = 0;
    int views_per_turn = 0;
    float start_angle_rad = 0.f;
    int rotation_direction = 1;
    float sid_mm = 0.f;
    float sdd_mm = 0.f;
    float start_z_mm = 0.f;
    float pitch_mm_per_turn = 0.f;
    float3 source_offset_mm = {0.f, 0.f, 0.f};
};

struct SFlatDetectorSpec {
    int channels = 0;
    int rows = 0;
    float channel_size_mm = 0.f;
    float row_size_mm = 0.f;
    SDetectorPoseSpec pose{};
};

// Cylindrical detector (declared for layout; rejected by this library).
struct SCylDetectorSpec {
    int channels = 0;
    int rows = 0;
    float channel_arc_mm = 0.f;
    float row_size_mm = 0.f;
    float curvature_radius_mm = 0.f;
    SDetectorPoseSpec pose{};
};

struct SVolumeGridSpec {
    int nx = 0;
    int ny = 0;
    int nz = 0;
    float voxel_x_mm = 0.f;
    float voxel_y_mm = 0.f;
    float voxel_z_mm = 0.f;
    float3 center_mm = {0.f, 0.f, 0.f};
};

// Volume rotation about its centre used only by the forward-projection
// pipeline (fixed world X, then Y, then Z; column-vector matrix Rz Ry Rx).
struct SForwardProjectionPose {
    bool enabled = false;
    float rotation_x_rad = 0.f;
    float rotation_y_rad = 0.f;
    float rotation_z_rad = 0.f;
};

struct SSystemConfig {
    EDetectorKind detector = EDetectorKind::Flat;
    ETrajectoryKind trajectory = ETrajectoryKind::Circular;
    SRegularCircularScanSpec circular{};
    SRegularHelicalScanSpec helical{};
    SFlatDetectorSpec flat_detector{};
    SCylDetectorSpec cylindrical_detector{};
    SVolumeGridSpec volume{};
    SForwardProjectionPose forward_projection_pose{};
};

// Non-standard trajectories (declared for layout; rejected by this library).
struct SPlanarSourceOrbitSpec {
    int total_views = 0;
    float start_angle_rad = 0.f;
    float scan_range_rad = 0.f;
    int rotation_direction = 1;
    float sid_mm = 0.f;
    float detector_y_mm = 0.f;
    float source_orbit_radius_mm = 0.f;
    float source_lateral_offset_mm = 0.f;
    int reconstruction_channels = 0;
    int reconstruction_rows = 0;
    EPlanarResampleMode resample_mode = EPlanarResampleMode::PerspectiveOrthogonal;
};

struct SNikonTiltedCtSpec {
    int total_views = 0;
    float start_angle_rad = 0.f;
    float scan_range_rad = 0.f;
    int rotation_direction = 1;
    float sid_mm = 0.f;
    float sdd_mm = 0.f;
    float tilt_rad = 0.f;
    float tilt_axis_azimuth_rad = 0.f;
    float3 source_offset_mm = {0.f, 0.f, 0.f};
    float3 rotation_axis_pivot_mm = {0.f, 0.f, 0.f};
};

struct SNonStandardGeometrySpec {
    SPlanarSourceOrbitSpec planar_source_orbit{};
    SNikonTiltedCtSpec nikon_tilted{};
};

// ----------------------------------------------------- algorithm params ---
struct SAnalyticFilterParams {
    EFdkFilter type = EFdkFilter::RamLak;
    float cutoff = .5f, gain = 1.f;  // cycles/sample; Nyquist is 0.5
    float butterworth_order = 2.f, kaiser_beta = 8.6f, tukey_alpha = .5f;
};

struct SParkerScanSpec {
    EParkerMode mode = EParkerMode::Auto;
};

struct SFdkAlgoParams {
    SParkerScanSpec parker{};
    SAnalyticFilterParams filter{};
};

// Parameters of the reference's iterative and helical algorithms (declared
// for layout; this library runs FDK and forward projection).
struct SIterAlgoParams {
    int iterations = 10;
    float relaxation = 1.f;
    int subsets = 1;
};

struct SCglsAlgoParams {
    int minimum_iterations = 0;
    int check_interval = 1;
    int patience = 1;
    float relative_residual = 0.f;
    bool robust_restart = true;
};

struct SPwlsAlgoParams {
    EPwlsRegularizerSpec regularizer = EPwlsRegularizerSpec::Quadratic;
    float regularization = 1e-3f;
    float huber_delta = 3e-3f;
    float epsilon = 1e-6f;
    float lower_bound = 0.f;
    float upper_bound = std::numeric_limits<float>::max();
    bool use_projection_weights = false;
};

struct STigreGradientAlgoParams {
    ETigreGradientMethodSpec method = ETigreGradientMethodSpec::OsSart;
    int block_size = 20;
    float lambda_reduction = 0.f;
    bool nesterov_relaxation = false;
    bool fdk_initialization = false;
    bool non_negative = true;
    int tv_iterations = 20;
    float tv_alpha = 0.002f;
    float tv_alpha_reduction = 0.95f;
    float maximum_update_ratio = 0.95f;
    float max_l2_error = -1.f;
};

struct SWfbpAlgoParams {
    float redundancy_flat = 0.6f;
    SAnalyticFilterParams filter{};
};

struct SReconstructionSpec {
    EPipeline pipeline = EPipeline::FDK;
    EForwardProjector forward_projector = EForwardProjector::Automatic;
    EBackProjector back_projector = EBackProjector::Automatic;
    SFdkAlgoParams fdk{};
    SIterAlgoParams iterative{};
    SCglsAlgoParams cgls{};
    SPwlsAlgoParams pwls{};
    STigreGradientAlgoParams tigre{};
    SWfbpAlgoParams wfbp{};
};

// Regularisation plugin of the reference's algebraic solvers (declared for
// layout; a plugin other than none is rejected here).
struct SAlgebraicRegularizationSpec {
    const char* plugin_id = nullptr;
    float strength = 0.f, huber_delta = 1e-3f, step_size = 0.f;
    int inner_iterations = 5, dimensions = 3;
    float epsilon = 1e-6f, strength_reduction = 1.f;
    bool non_negative = true;
};

// Statistical reconstruction (declared for layout; rejected here).
struct SDataFidelitySpec {
    EDataFidelityKind kind = EDataFidelityKind::WeightedLeastSquares;
    bool use_projection_weights = false;
    bool normalize_by_ray_count = false;
    bool require_verified_adjoint = false;
    float scale = 1.f;
};

struct SStatisticalRegularizationSpec {
    const char* plugin_id = "huber_tv_prox";
    float strength = 0.f;
    float shape = 1e-3f;
    int dimensions = 3;
};

struct SStatisticalOptimizerSpec {
    EStatisticalOptimizer kind = EStatisticalOptimizer::RegularizedAlgebraic;
    int iterations = 10;
    float step_size = 0.f;
    bool backtracking = true;
    int max_backtracking = 20;
    float step_shrink = 0.5f;
    float relative_tolerance = 0.f;
    int minimum_iterations = 1;
};

struct SStatisticalConstraintSpec {
    float lower_bound = 0.f;
    float upper_bound = std::numeric_limits<float>::max();
};

struct SStatisticalReconstructionSpec {
    SDataFidelitySpec data_fidelity{};
    SStatisticalRegularizationSpec regularization{};
    SStatisticalOptimizerSpec optimizer{};
    SStatisticalConstraintSpec constraints{};
};

// ------------------------------------------------------------ the session ---
struct SSystemSpec {
    uint32_t struct_size = sizeof(SSystemSpec);
    uint32_t api_version = 2;
    SSystemConfig geometry{};
    SReconstructionSpec reconstruction{};
    int device = 0;
    // Optional tails, each read only when struct_size covers it whole (a
    // partly covered tail is InvalidConfig).
    SNonStandardGeometrySpec nonstandard{};
    SAlgebraicRegularizationSpec regularization{};
    SStatisticalReconstructionSpec statistical{};
    // Caller geometry for a flat detector: flat_frame_count views (the
    // scan's total_views), borrowed only during initialize.  detS is pixel
    // (0,0), detU/detV are one-pixel steps, angle.x the view angle.  FDK
    // accepts frames within 1e-3 of the nominal orbit (then uses them);
    // ForwardProjection accepts any finite frames with orthogonal detU, detV.
    const SConeProjGeomVec* flat_frames = nullptr;
    int flat_frame_count = 0;
};

// Fills a host destination with the requested views, [view][v][u] (the
// reference's projection reader; not accepted by FDK or forward projection).
using ProjectionReadCallback = bool (*)(void*, const int*, int, float*, size_t);

// Contiguous float arrays: projection [view][v][u], volume [z][y][x].
struct Buffer {
    float* data = nullptr;
    EMemoryLocation location = EMemoryLocation::Device;
    size_t element_count = 0;
};

struct SExecutionRequest {
    uint32_t struct_size = sizeof(SExecutionRequest);
    uint32_t api_version = 2;
    Buffer projection{};
    Buffer volume{};
    int view_offset = 0;
    int view_count = 0;        // 0: all prepared views
    bool clear_output = true;  // FDK: only the first batch of a sequence
    int iteration_count = 0;
    // called on execute's thread after the GPU work; must not throw
    void (*progress_callback)(void*, int completed, int total) = nullptr;
    void* progress_user_data = nullptr;
    // projection reader and statistical weights of the reference's iterative
    // pipelines (a reader or weights make FDK / forward projection return
    // UnsupportedCombination, as the reference's do)
    ProjectionReadCallback projection_read = nullptr;
    void* projection_read_user_data = nullptr;
    int projection_batch_views = 64;
    int projection_batch_mib = 256;
    Buffer projection_weights{};
    ProjectionReadCallback projection_weights_read = nullptr;
    void* projection_weights_read_user_data = nullptr;
};

class YKB_SESSION_API IReconstructionSession {
public:
    virtual ~IReconstructionSession() = default;
    virtual bool initialize(const SSystemSpec& system) = 0;
    virtual bool execute(const SExecutionRequest& request) = 0;
    virtual bool isInitialized() const = 0;
    virtual EApiErrorCode lastError() const = 0;
    virtual const char* lastErrorMessage() const = 0;
    virtual void reset() = 0;
    virtual void release() = 0;
};

struct YKB_SESSION_API ReconstructionSessionFactory {
    static IReconstructionSession* create();
    static void destroy(IReconstructionSession* session);
};

} // namespace YK
