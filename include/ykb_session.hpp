// ykb_session.hpp -- C++ Session layer of libykb for the flat-panel circular
// path: the names, members, defaults and error behaviour of YKCBCT's public
// API (include/YKCBCT/interface/YkReconstructionApi.hpp:18-98,
// YkReconstructionTypes.hpp, YkSystemReconstruction.hpp, and the geometry
// specs of include/YKCBCT/geometry/YkGeometryBuilderTypes.hpp), so code
// written against that API for FDK and forward projection compiles and runs
// unchanged on this library.
//
// Scope: flat detector, circular trajectory, EPipeline::FDK and
// EPipeline::ForwardProjection with EForwardProjector::Joseph, ::Siddon or
// ::Automatic (Siddon for a flat detector, as the reference resolves it).  Other
// pipelines, detectors and trajectories are outside this library and are
// rejected with EApiErrorCode::UnsupportedCombination at initialize().
// Members the reference carries only for those other algorithms (helical and
// cylindrical specs, iterative/statistical/regularisation tails, projection
// readers) are not declared here.
//
// This is a source-level interface over the C-ABI of ykb.h (the binary
// boundary); every execute() runs on the session's own CUDA stream and
// returns after the GPU work completes, as the reference's does.
#pragma once

#include <cstddef>
#include <cstdint>

#include <vector_types.h>  // float3, as the reference's public headers use

#if defined(_WIN32)
#define YKB_SESSION_API __declspec(dllexport)
#else
#define YKB_SESSION_API __attribute__((visibility("default")))
#endif

namespace YK {

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

enum class EApiErrorCode : int32_t {
    None = 0, InvalidConfig, InvalidGeometry, UnsupportedCombination, AlgorithmUnderTest,
    InvalidBuffer, StreamingStateError, CudaError,
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

struct SFlatDetectorSpec {
    int channels = 0;
    int rows = 0;
    float channel_size_mm = 0.f;
    float row_size_mm = 0.f;
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
    SFlatDetectorSpec flat_detector{};
    SVolumeGridSpec volume{};
    SForwardProjectionPose forward_projection_pose{};
};

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

struct SReconstructionSpec {
    EPipeline pipeline = EPipeline::FDK;
    EForwardProjector forward_projector = EForwardProjector::Automatic;
    EBackProjector back_projector = EBackProjector::Automatic;
    SFdkAlgoParams fdk{};
};

struct SSystemSpec {
    uint32_t struct_size = sizeof(SSystemSpec);
    uint32_t api_version = 2;
    SSystemConfig geometry{};
    SReconstructionSpec reconstruction{};
    int device = 0;
};

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
