// Exercises libykb's C++ Session layer the way YKCBCT's own tests use its
// Session (unit_test/test_small_reconstruction.cpp, dlltest/test_shepp_logan.cpp).
// Built and run by tests/test_session.py.
//
//   session_test validate                       error codes (no GPU needed)
//   session_test roundtrip                      FP(Joseph) -> FDK on a small grid
//   session_test streaming                      full vs 47-view batches, streaming errors
//   session_test fdk <proj.f32> <vol.f32> ...   FDK of a projection file (parity)
//   session_test fp  <vol.f32> <proj.f32> ...   Joseph FP of a volume file (parity)
//   session_test fdk|fp ... <frames.bin>        the same with caller geometry
//                                               (SSystemSpec::flat_frames)
//   session_test frames                         caller frames equal to the orbit
//                                               vs the orbit; request tails
// Prints one JSON object per mode; exit code 0 when the mode's checks pass.
#include "ykb_session.hpp"
#include "ykb.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace YK;

namespace {

using SessionPtr = std::unique_ptr<IReconstructionSession, decltype(&ReconstructionSessionFactory::destroy)>;

SessionPtr make_session()
{
    return SessionPtr(ReconstructionSessionFactory::create(), &ReconstructionSessionFactory::destroy);
}

// unit_test/test_small_reconstruction.cpp:26-45 geometry
SSystemSpec small_system(EPipeline pipeline)
{
    SSystemSpec s{};
    s.geometry.detector = EDetectorKind::Flat;
    s.geometry.trajectory = ETrajectoryKind::Circular;
    s.geometry.circular.total_views = 96;
    s.geometry.circular.views_per_turn = 96;
    s.geometry.circular.sid_mm = 100.f;
    s.geometry.circular.sdd_mm = 200.f;
    s.geometry.flat_detector.channels = 48;
    s.geometry.flat_detector.rows = 32;
    s.geometry.flat_detector.channel_size_mm = 1.f;
    s.geometry.flat_detector.row_size_mm = 1.f;
    s.geometry.volume = {24, 24, 16, 1.f, 1.f, 1.f, {0.f, 0.f, 0.f}};
    s.reconstruction.pipeline = pipeline;
    s.reconstruction.forward_projector = EForwardProjector::Joseph;
    s.reconstruction.back_projector = EBackProjector::JosephV3;
    s.reconstruction.fdk.filter.type = EFdkFilter::RamLak;
    return s;
}

// the scan's own orbit as caller frames, from libykb's builder (the
// reference's buildSystemGeometry gives the same floats)
std::vector<SConeProjGeomVec> nominal_frames(const SSystemSpec& s)
{
    const auto& c = s.geometry.circular;
    const auto& d = s.geometry.flat_detector;
    ykb_circular_flat spec{};
    spec.total_views = c.total_views;
    spec.views_per_turn = c.views_per_turn;
    spec.start_angle_rad = c.start_angle_rad;
    spec.rotation_direction = c.rotation_direction;
    spec.sid_mm = c.sid_mm;
    spec.sdd_mm = c.sdd_mm;
    spec.z_mm = c.z_mm;
    spec.channels = d.channels;
    spec.rows = d.rows;
    spec.channel_size_mm = d.channel_size_mm;
    spec.row_size_mm = d.row_size_mm;
    std::vector<SConeProjGeomVec> out(static_cast<size_t>(c.total_views));
    if (ykb_build_circular_flat(&spec, reinterpret_cast<ykb_cone_view*>(out.data()), c.total_views) != YKB_OK)
        out.clear();
    return out;
}

std::vector<float> analytic_phantom(const SVolumeGridSpec& g)
{
    std::vector<float> v(static_cast<size_t>(g.nx) * g.ny * g.nz, 0.f);
    for (int z = 0; z < g.nz; ++z)
        for (int y = 0; y < g.ny; ++y)
            for (int x = 0; x < g.nx; ++x) {
                const float px = (x + 0.5f - 0.5f * g.nx) * g.voxel_x_mm;
                const float py = (y + 0.5f - 0.5f * g.ny) * g.voxel_y_mm;
                const float pz = (z + 0.5f - 0.5f * g.nz) * g.voxel_z_mm;
                float value = px * px / 49.f + py * py / 64.f + pz * pz / 25.f <= 1.f ? 0.02f : 0.f;
                if ((px - 3.f) * (px - 3.f) + (py + 2.f) * (py + 2.f) + pz * pz <= 2.25f) value = 0.06f;
                v[(static_cast<size_t>(z) * g.ny + y) * g.nx + x] = value;
            }
    return v;
}

Buffer host(std::vector<float>& v) { return {v.data(), EMemoryLocation::Host, v.size()}; }

double cosine(const std::vector<float>& a, const std::vector<float>& b)
{
    double p = 0, ea = 0, eb = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        p += double(a[i]) * b[i];
        ea += double(a[i]) * a[i];
        eb += double(b[i]) * b[i];
    }
    return p / std::sqrt(std::max(ea * eb, 1e-30));
}

int expect_code(const char* name, bool ok, IReconstructionSession& s, EApiErrorCode want, int& failures)
{
    const bool pass = !ok && s.lastError() == want && s.lastErrorMessage()[0] != 0;
    std::printf("\"%s\": %s, ", name, pass ? "true" : "false");
    if (!pass) {
        ++failures;
        std::fprintf(stderr, "%s: ok=%d code=%d msg=%s\n", name, ok, int(s.lastError()), s.lastErrorMessage());
    }
    return pass;
}

int mode_validate()
{
    int failures = 0;
    std::printf("{");
    auto s = make_session();
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.api_version = 1;
        expect_code("api_version", s->initialize(spec), *s, EApiErrorCode::InvalidConfig, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.struct_size = 8;
        expect_code("truncated", s->initialize(spec), *s, EApiErrorCode::InvalidConfig, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.geometry.detector = EDetectorKind::Cylindrical;
        expect_code("cylindrical", s->initialize(spec), *s, EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.geometry.trajectory = ETrajectoryKind::Helical;
        expect_code("helical", s->initialize(spec), *s, EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::CGLS);
        expect_code("cgls", s->initialize(spec), *s, EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::ForwardProjection);
        spec.reconstruction.forward_projector = EForwardProjector::SeparableFootprint;
        expect_code("fp_footprint", s->initialize(spec), *s, EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::ForwardProjection);
        spec.geometry.forward_projection_pose.rotation_x_rad = NAN;
        expect_code("pose_nan", s->initialize(spec), *s, EApiErrorCode::InvalidGeometry, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.geometry.volume.nx = 0;
        expect_code("volume", s->initialize(spec), *s, EApiErrorCode::InvalidGeometry, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.geometry.circular.sdd_mm = 50.f;
        expect_code("sdd", s->initialize(spec), *s, EApiErrorCode::InvalidGeometry, failures);
    }
    // caller-frame tail (src/interface/YkReconstructionApi.cpp:144-168)
    std::vector<SConeProjGeomVec> orbit = nominal_frames(small_system(EPipeline::FDK));
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.struct_size = static_cast<uint32_t>(offsetof(SSystemSpec, flat_frames) + 4);
        expect_code("frame_tail_truncated", s->initialize(spec), *s, EApiErrorCode::InvalidConfig, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.flat_frame_count = 5;
        expect_code("frame_count_no_buffer", s->initialize(spec), *s, EApiErrorCode::InvalidConfig, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::PWLS);
        spec.flat_frames = orbit.data();
        spec.flat_frame_count = static_cast<int>(orbit.size());
        expect_code("frames_pwls", s->initialize(spec), *s, EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.flat_frames = orbit.data();
        spec.flat_frame_count = static_cast<int>(orbit.size()) - 1;
        expect_code("fdk_frames_count", s->initialize(spec), *s, EApiErrorCode::InvalidGeometry, failures);
    }
    {
        std::vector<SConeProjGeomVec> off = orbit;
        off[7].detS.x += 0.01f;  // 10 um off the orbit, beyond the 1e-3 mm the FDK accepts
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.flat_frames = off.data();
        spec.flat_frame_count = static_cast<int>(off.size());
        expect_code("fdk_frames_off_orbit", s->initialize(spec), *s,
            EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        std::vector<SConeProjGeomVec> skew = orbit;
        skew[3].detV.x += 0.1f;  // detU and detV no longer orthogonal
        SSystemSpec spec = small_system(EPipeline::ForwardProjection);
        spec.flat_frames = skew.data();
        spec.flat_frame_count = static_cast<int>(skew.size());
        expect_code("fp_frames_skewed", s->initialize(spec), *s, EApiErrorCode::InvalidGeometry, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.regularization.plugin_id = "huber_tv_prox";
        expect_code("regularization_plugin", s->initialize(spec), *s,
            EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        SSystemSpec spec = small_system(EPipeline::FDK);
        spec.struct_size = static_cast<uint32_t>(offsetof(SSystemSpec, statistical) + 4);
        expect_code("statistical_tail_truncated", s->initialize(spec), *s,
            EApiErrorCode::InvalidConfig, failures);
    }
    {
        std::vector<float> a(10), b(10);
        SExecutionRequest req{};
        req.projection = host(a);
        req.volume = host(b);
        expect_code("not_initialized", s->execute(req), *s, EApiErrorCode::StreamingStateError, failures);
    }
    std::printf("\"failures\": %d}\n", failures);
    return failures == 0 ? 0 : 1;
}

int mode_roundtrip()
{
    auto spec = small_system(EPipeline::ForwardProjection);
    auto truth = analytic_phantom(spec.geometry.volume);
    std::vector<float> proj(48 * 32 * 96, 0.f), rec(truth.size(), 0.f);
    auto fp = make_session();
    if (!fp->initialize(spec)) { std::fprintf(stderr, "fp init: %s\n", fp->lastErrorMessage()); return 2; }
    SExecutionRequest req{};
    req.volume = host(truth);
    req.projection = host(proj);
    req.view_count = 96;
    if (!fp->execute(req)) { std::fprintf(stderr, "fp: %s\n", fp->lastErrorMessage()); return 2; }
    bool nonneg = true;
    float pmax = 0.f;
    for (float p : proj) { nonneg &= std::isfinite(p) && p >= 0.f; pmax = std::max(pmax, p); }
    spec.reconstruction.pipeline = EPipeline::FDK;
    auto fdk = make_session();
    if (!fdk->initialize(spec)) { std::fprintf(stderr, "fdk init: %s\n", fdk->lastErrorMessage()); return 2; }
    req.volume = host(rec);
    if (!fdk->execute(req)) { std::fprintf(stderr, "fdk: %s\n", fdk->lastErrorMessage()); return 2; }
    float rmax = -1e30f;
    bool finite = true;
    for (float r : rec) { finite &= std::isfinite(r); rmax = std::max(rmax, r); }
    const double c = cosine(truth, rec);
    std::printf("{\"cosine\": %.6f, \"proj_nonneg\": %s, \"proj_max\": %.6f, \"rec_max\": %.6f}\n", c,
        nonneg ? "true" : "false", pmax, rmax);
    return (nonneg && pmax > 0.f && finite && rmax > 0.f && c > 0.70) ? 0 : 1;
}

// dlltest/test_shepp_logan.cpp geometry (64^3 @ 0.75, 128^2 @ 0.8, 360 views,
// SID/SDD 200/400) with the analytic phantom scaled to the grid; full run vs
// 47-view streamed batches (pin: max diff < 1e-5), plus the streaming errors.
int mode_streaming()
{
    SSystemSpec spec{};
    spec.geometry.circular.total_views = 360;
    spec.geometry.circular.views_per_turn = 360;
    spec.geometry.circular.sid_mm = 200.f;
    spec.geometry.circular.sdd_mm = 400.f;
    spec.geometry.flat_detector.channels = 128;
    spec.geometry.flat_detector.rows = 128;
    spec.geometry.flat_detector.channel_size_mm = 0.8f;
    spec.geometry.flat_detector.row_size_mm = 0.8f;
    spec.geometry.volume = {64, 64, 64, 0.75f, 0.75f, 0.75f, {0.f, 0.f, 0.f}};
    spec.reconstruction.pipeline = EPipeline::ForwardProjection;
    spec.reconstruction.forward_projector = EForwardProjector::Joseph;
    auto truth = analytic_phantom(spec.geometry.volume);
    const size_t view_elems = 128 * 128;
    std::vector<float> proj(view_elems * 360);
    auto fp = make_session();
    if (!fp->initialize(spec)) return 2;
    SExecutionRequest req{};
    req.volume = host(truth);
    req.projection = host(proj);
    if (!fp->execute(req)) { std::fprintf(stderr, "fp: %s\n", fp->lastErrorMessage()); return 2; }

    spec.reconstruction.pipeline = EPipeline::FDK;
    auto full = make_session();
    if (!full->initialize(spec)) return 2;
    std::vector<float> a(truth.size()), b(truth.size(), 7.f);
    req.volume = host(a);
    if (!full->execute(req)) { std::fprintf(stderr, "full: %s\n", full->lastErrorMessage()); return 2; }

    auto streamed = make_session();
    if (!streamed->initialize(spec)) return 2;
    int failures = 0;
    std::printf("{");
    for (int offset = 0; offset < 360; offset += 47) {
        SExecutionRequest batch{};
        batch.view_offset = offset;
        batch.view_count = std::min(47, 360 - offset);
        batch.projection = {proj.data() + view_elems * offset, EMemoryLocation::Host,
            view_elems * batch.view_count};
        batch.volume = host(b);
        batch.clear_output = offset == 0;
        if (offset == 47) {
            SExecutionRequest again = batch;
            again.view_offset = 0;
            expect_code("repeat_batch", streamed->execute(again), *streamed,
                EApiErrorCode::StreamingStateError, failures);
            SExecutionRequest clear = batch;
            clear.clear_output = true;
            expect_code("clear_later", streamed->execute(clear), *streamed,
                EApiErrorCode::StreamingStateError, failures);
            SExecutionRequest small = batch;
            small.projection.element_count = 5;
            expect_code("element_count", streamed->execute(small), *streamed,
                EApiErrorCode::InvalidBuffer, failures);
        }
        if (!streamed->execute(batch)) { std::fprintf(stderr, "batch: %s\n", streamed->lastErrorMessage()); return 2; }
    }
    double max_diff = 0.0;
    for (size_t i = 0; i < a.size(); ++i) max_diff = std::max(max_diff, double(std::fabs(a[i] - b[i])));
    const double c = cosine(truth, a);
    double num = 0, den = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        num += double(a[i] - truth[i]) * (a[i] - truth[i]);
        den += double(truth[i]) * truth[i];
    }
    const double nrmse = std::sqrt(num / std::max(den, 1e-30));
    std::printf("\"max_diff\": %.3e, \"cosine\": %.6f, \"nrmse\": %.6f, \"failures\": %d}\n", max_diff, c,
        nrmse, failures);
    return (failures == 0 && max_diff < 1e-5 && c > 0.85 && nrmse < 0.65) ? 0 : 1;
}

std::vector<float> read_f32(const char* path, size_t n)
{
    std::vector<float> v(n);
    FILE* f = std::fopen(path, "rb");
    if (!f || std::fread(v.data(), sizeof(float), n, f) != n) { std::fprintf(stderr, "read %s\n", path); std::exit(3); }
    std::fclose(f);
    return v;
}

void write_f32(const char* path, const std::vector<float>& v)
{
    FILE* f = std::fopen(path, "wb");
    if (!f || std::fwrite(v.data(), sizeof(float), v.size(), f) != v.size()) { std::fprintf(stderr, "write %s\n", path); std::exit(3); }
    std::fclose(f);
}

// fdk|fp <in> <out> views per_turn sid sdd nu nv du dv nx ny nz vox filter [frames]
// frames: a file of `views` SConeProjGeomVec records passed as flat_frames
int mode_file(bool fdk, int argc, char** argv, bool siddon = false)
{
    if (argc < 17) return 4;
    SSystemSpec spec{};
    spec.geometry.circular.total_views = std::atoi(argv[4]);
    spec.geometry.circular.views_per_turn = std::atoi(argv[5]);
    spec.geometry.circular.sid_mm = std::atof(argv[6]);
    spec.geometry.circular.sdd_mm = std::atof(argv[7]);
    spec.geometry.flat_detector.channels = std::atoi(argv[8]);
    spec.geometry.flat_detector.rows = std::atoi(argv[9]);
    spec.geometry.flat_detector.channel_size_mm = std::atof(argv[10]);
    spec.geometry.flat_detector.row_size_mm = std::atof(argv[11]);
    const float vox = std::atof(argv[15]);
    spec.geometry.volume = {std::atoi(argv[12]), std::atoi(argv[13]), std::atoi(argv[14]), vox, vox, vox,
        {0.f, 0.f, 0.f}};
    spec.reconstruction.pipeline = fdk ? EPipeline::FDK : EPipeline::ForwardProjection;
    // the FP modes pick the projector: "fp" Joseph, "fp_auto" Automatic (Siddon)
    spec.reconstruction.forward_projector = siddon ? EForwardProjector::Automatic
                                                   : EForwardProjector::Joseph;
    spec.reconstruction.fdk.filter.type = static_cast<EFdkFilter>(std::atoi(argv[16]));
    const size_t pn = size_t(spec.geometry.circular.total_views) * spec.geometry.flat_detector.channels *
        spec.geometry.flat_detector.rows;
    const size_t vn = size_t(spec.geometry.volume.nx) * spec.geometry.volume.ny * spec.geometry.volume.nz;
    std::vector<float> frame_floats;
    if (argc > 17) {
        frame_floats = read_f32(argv[17], size_t(spec.geometry.circular.total_views) * 20);
        spec.flat_frames = reinterpret_cast<const SConeProjGeomVec*>(frame_floats.data());
        spec.flat_frame_count = spec.geometry.circular.total_views;
    }
    auto s = make_session();
    if (!s->initialize(spec)) { std::fprintf(stderr, "init: %s\n", s->lastErrorMessage()); return 2; }
    std::vector<float> proj = fdk ? read_f32(argv[2], pn) : std::vector<float>(pn);
    std::vector<float> vol = fdk ? std::vector<float>(vn) : read_f32(argv[2], vn);
    SExecutionRequest req{};
    req.projection = host(proj);
    req.volume = host(vol);
    if (!s->execute(req)) { std::fprintf(stderr, "execute: %s\n", s->lastErrorMessage()); return 2; }
    write_f32(argv[3], fdk ? vol : proj);
    std::printf("{\"ok\": true}\n");
    return 0;
}

// Joseph FP through caller frames equal to the scan's orbit against FP of the
// orbit itself (max difference < 1e-5, the reference's framework/
// external-geometry pin, Yktest/test_pipeline_smoke.cpp:2029-2075), and the
// request tails the reference's iterative pipelines own (a projection reader
// or statistical weights make forward projection return UnsupportedCombination)
int mode_frames()
{
    SSystemSpec spec = small_system(EPipeline::ForwardProjection);
    const auto truth = analytic_phantom(spec.geometry.volume);
    std::vector<float> vol = truth;
    const size_t pn = size_t(48) * 32 * 96;
    std::vector<float> a(pn), b(pn);
    SExecutionRequest req{};
    req.volume = host(vol);
    req.projection = host(a);
    auto orbit_session = make_session();
    if (!orbit_session->initialize(spec) || !orbit_session->execute(req)) {
        std::fprintf(stderr, "orbit: %s\n", orbit_session->lastErrorMessage());
        return 2;
    }
    const std::vector<SConeProjGeomVec> frames = nominal_frames(spec);
    spec.flat_frames = frames.data();
    spec.flat_frame_count = static_cast<int>(frames.size());
    auto frame_session = make_session();
    req.projection = host(b);
    if (!frame_session->initialize(spec) || !frame_session->execute(req)) {
        std::fprintf(stderr, "frames: %s\n", frame_session->lastErrorMessage());
        return 2;
    }
    double max_diff = 0.0;
    for (size_t i = 0; i < pn; ++i) max_diff = std::max(max_diff, double(std::fabs(a[i] - b[i])));
    int failures = 0;
    std::printf("{");
    {
        SExecutionRequest r = req;
        r.projection_read = [](void*, const int*, int, float*, size_t) { return true; };
        expect_code("projection_reader", frame_session->execute(r), *frame_session,
            EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        SExecutionRequest r = req;
        r.projection_weights = host(a);
        expect_code("projection_weights", frame_session->execute(r), *frame_session,
            EApiErrorCode::UnsupportedCombination, failures);
    }
    {
        SExecutionRequest r = req;
        r.struct_size = static_cast<uint32_t>(offsetof(SExecutionRequest, projection_read) + 4);
        expect_code("source_tail_truncated", frame_session->execute(r), *frame_session,
            EApiErrorCode::InvalidConfig, failures);
    }
    std::printf("\"max_diff\": %.3e, \"failures\": %d}\n", max_diff, failures);
    return (failures == 0 && max_diff < 1e-5) ? 0 : 1;
}

} // namespace

int main(int argc, char** argv)
{
    const std::string mode = argc > 1 ? argv[1] : "";
    if (mode == "validate") return mode_validate();
    if (mode == "roundtrip") return mode_roundtrip();
    if (mode == "streaming") return mode_streaming();
    if (mode == "fdk") return mode_file(true, argc, argv);
    if (mode == "fp") return mode_file(false, argc, argv);
    if (mode == "fp_auto") return mode_file(false, argc, argv, true);
    if (mode == "frames") return mode_frames();
    std::fprintf(stderr, "usage: session_test validate|roundtrip|streaming|frames|fdk|fp|fp_auto ...\n");
    return 4;
}
