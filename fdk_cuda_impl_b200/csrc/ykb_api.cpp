// C-ABI entry points of libykb.so (declared in include/ykb.h).
#include "ykb_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>

namespace ykb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
const char* last_error() { return g_last_error.c_str(); }

ykb_status cuda_status(cudaError_t status, const char* what)
{
    if (status == cudaSuccess) return YKB_OK;
    set_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorName(status) + " (" +
        cudaGetErrorString(status) + ")");
    if (status == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // allocation failure is not sticky; clear it
        return YKB_ERR_OUT_OF_MEMORY;
    }
    return YKB_ERR_CUDA;
}

namespace {

ykb_status fail(ykb_status code, const std::string& msg)
{
    set_error(msg);
    return code;
}

bool valid_volume(const ykb_volume* v)
{
    return v && v->nx > 0 && v->ny > 0 && v->nz > 0 && v->vox_x > 0.f && v->vox_y > 0.f &&
        v->vox_z > 0.f && std::isfinite(v->vox_x) && std::isfinite(v->vox_y) &&
        std::isfinite(v->vox_z) && std::isfinite(v->center_x) && std::isfinite(v->center_y) &&
        std::isfinite(v->center_z);
}

// validAnalyticFilter (src/Filter/YkAnalyticFilterSettings.hpp:5-13)
bool valid_filter(const ykb_filter* p)
{
    return p && p->type >= 0 && p->type <= 9 && std::isfinite(p->cutoff) && p->cutoff > 0.f &&
        p->cutoff <= 0.5f && std::isfinite(p->gain) && p->gain > 0.f &&
        std::isfinite(p->butterworth_order) && p->butterworth_order > 0.f &&
        std::isfinite(p->kaiser_beta) && p->kaiser_beta >= 0.f && std::isfinite(p->tukey_alpha) &&
        p->tukey_alpha >= 0.f && p->tukey_alpha <= 1.f;
}

ykb_status check_device(int device)
{
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetDeviceCount");
    if (device < 0 || device >= count)
        return fail(YKB_ERR_INVALID_CONFIG, "device index out of range");
    return YKB_OK;
}

size_t volume_elems(const ykb_volume& v)
{
    return static_cast<size_t>(v.nx) * v.ny * v.nz;
}

// Views per workspace chunk: bounded so the filter workspace stays below
// about 8 GiB whatever the scan length.  a_bytes: bytes per pixel of the
// preweighted rows (4 as float or as two BF16 parts, 6 as three).
int chunk_capacity(int n_views, int nu, int nv, int a_bytes)
{
    // preweighted rows + filtered tap pairs (8 B) per detector pixel
    const size_t per_view = static_cast<size_t>(nu) * nv * (a_bytes + 8);
    const size_t budget = size_t(8) << 30;
    const size_t cap = std::max<size_t>(1, budget / std::max<size_t>(per_view, 1));
    return static_cast<int>(std::min<size_t>(n_views, cap));
}

} // namespace
} // namespace ykb

using namespace ykb;

extern "C" {

YKB_API int ykb_version(void) { return 100; }

YKB_API const char* ykb_last_error(void) { return ykb::last_error(); }

// include/YKCBCT/interface/YkSystemReconstruction.hpp:22-28
YKB_API float ykb_regular_scan_range(int total_views, int views_per_turn)
{
    constexpr float kTwoPi = 6.28318530717958647692f;
    return kTwoPi * static_cast<float>(total_views) / static_cast<float>(views_per_turn);
}

YKB_API ykb_status ykb_build_circular_flat(const ykb_circular_flat* spec, ykb_cone_view* out,
    int capacity)
{
    clear_error();
    if (!spec || !out) return fail(YKB_ERR_INVALID_BUFFER, "null spec or output");
    if (capacity < spec->total_views)
        return fail(YKB_ERR_INVALID_BUFFER, "output capacity smaller than total_views");
    std::string why;
    if (!build_circular_flat(*spec, out, why)) return fail(YKB_ERR_INVALID_GEOMETRY, why);
    return YKB_OK;
}

// ------------------------------------------------------------------ FDK ---
YKB_API ykb_status ykb_fdk_plan_create(const ykb_cone_view* views, int n_views, int nu, int nv,
    float scan_range_rad, const ykb_volume* volume, const ykb_filter* filter, int precision,
    int device, ykb_fdk_plan** plan_out)
{
    return ykb_fdk_plan_create_ex(views, n_views, nu, nv, scan_range_rad, 0.f, 1, volume, filter,
        precision, YKB_PARKER_DISABLED, device, plan_out);
}

YKB_API ykb_status ykb_fdk_plan_create_ex(const ykb_cone_view* views, int n_views, int nu, int nv,
    float scan_range_rad, float start_angle_rad, int rotation_direction, const ykb_volume* volume,
    const ykb_filter* filter, int precision, int parker_mode, int device, ykb_fdk_plan** plan_out)
{
    clear_error();
    if (!plan_out) return fail(YKB_ERR_INVALID_BUFFER, "null plan output");
    if (parker_mode != YKB_PARKER_AUTO && parker_mode != YKB_PARKER_DISABLED &&
        parker_mode != YKB_PARKER_ENABLED)
        return fail(YKB_ERR_INVALID_CONFIG, "unknown Parker mode");
    if (rotation_direction != 1 && rotation_direction != -1)
        return fail(YKB_ERR_INVALID_CONFIG, "rotation direction must be +1 or -1");
    *plan_out = nullptr;
    if (!views || n_views <= 0 || nu <= 0 || nv <= 0)
        return fail(YKB_ERR_INVALID_CONFIG, "views, view count and detector size must be positive");
    if (!valid_volume(volume)) return fail(YKB_ERR_INVALID_CONFIG, "invalid volume grid");
    if (!valid_filter(filter)) return fail(YKB_ERR_INVALID_CONFIG, "invalid analytic filter parameters");
    if (precision != YKB_PRECISION_FP32 && precision != YKB_PRECISION_BF16)
        return fail(YKB_ERR_INVALID_CONFIG, "unknown precision");
    if (const ykb_status st = check_device(device)) return st;
    DeviceGuard guard(device);

    ykb_fdk_plan* p = new (std::nothrow) ykb_fdk_plan();
    if (!p) return fail(YKB_ERR_OUT_OF_MEMORY, "host allocation failed");
    p->device = device; p->n_views = n_views; p->nu = nu; p->nv = nv;
    p->scan_range = scan_range_rad; p->volume = *volume; p->filter = *filter;
    p->precision = precision;
    std::string why;
    if (!derive_fdk_geometry(views, n_views, nu, nv, scan_range_rad, p->derived, why)) {
        delete p;
        return fail(YKB_ERR_INVALID_GEOMETRY, why);
    }
    // Parker weighting: Enabled, or Auto on a short scan
    // (include/YKCBCT/interface/YkSystemReconstruction.hpp:29-39)
    const bool parker = parker_mode == YKB_PARKER_ENABLED ||
        (parker_mode == YKB_PARKER_AUTO && scan_range_rad < 6.28318530717958647692f - 1e-5f);
    std::vector<float> parker_w;
    if (parker && !build_parker_weights(p->derived, views, nu, nv, scan_range_rad,
            start_angle_rad, rotation_direction, parker_w, why)) {
        delete p;
        return fail(YKB_ERR_INVALID_GEOMETRY, why);
    }
    std::vector<FdkViewCoef> coef;
    std::vector<FdkPreweightView> pw;
    build_fdk_coefficients(p->derived, nu, coef, pw, p->axial);
    // weights are built once with du of the first view (.../FDK/
    // YkFDKFilterProcessor.hpp:111,216-232)
    std::vector<double> h;
    build_ramp_kernel(nu, p->derived[0].du, *filter, h);
    std::vector<float> hf(h.begin(), h.end());

    // the ramp filter runs on the tensor cores: BF16 plans with two BF16
    // parts per operand, FP32 plans with three (FP32 accuracy); the FP32
    // Toeplitz product on the CUDA cores when tcgen05 is unavailable, or
    // when YKB_FDK_FILTER=simt asks for it (tests compare the two)
    const char* filter_path = std::getenv("YKB_FDK_FILTER");
    const bool force_simt = filter_path && std::strcmp(filter_path, "simt") == 0;
    p->tc_filter = tcgen05_filter_supported(nu) &&
        (precision == YKB_PRECISION_BF16 || !force_simt);
    p->tc_parts = p->tc_filter ? (precision == YKB_PRECISION_BF16 ? 2 : 3) : 0;
    p->lda = p->tc_filter ? tc_filter_lda(nu) : nu;
    const int a_bytes = p->tc_parts == 3 ? 6 : 4;
    p->batch_capacity = chunk_capacity(n_views, nu, nv, a_bytes);
    // work_a holds the preweighted rows: float, or the bf16 parts in turn
    const size_t chunk_elems = static_cast<size_t>(p->batch_capacity) * p->lda * nv;
    cudaError_t e;
    if ((e = p->coef.alloc(sizeof(FdkViewCoef) * n_views)) != cudaSuccess ||
        (e = p->pwv.alloc(sizeof(FdkPreweightView) * n_views)) != cudaSuccess ||
        (e = p->ramp.alloc(sizeof(float) * hf.size())) != cudaSuccess ||
        (e = p->err_flag.alloc(4 * sizeof(int))) != cudaSuccess ||
        (e = p->work_a.alloc(chunk_elems * a_bytes)) != cudaSuccess) {
        delete p;
        return cuda_status(e, "cudaMalloc (FDK plan workspace)");
    }
    if ((e = cudaMemcpy(p->coef.ptr, coef.data(), sizeof(FdkViewCoef) * n_views,
             cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(p->pwv.ptr, pw.data(), sizeof(FdkPreweightView) * n_views,
             cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(p->ramp.ptr, hf.data(), sizeof(float) * hf.size(),
             cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(p->err_flag.ptr, 0, 4 * sizeof(int))) != cudaSuccess) {
        delete p;
        return cuda_status(e, "cudaMemcpy (FDK plan tables)");
    }
    if (!parker_w.empty() &&
        ((e = p->parker.alloc(parker_w.size() * sizeof(float))) != cudaSuccess ||
         (e = cudaMemcpy(p->parker.ptr, parker_w.data(), parker_w.size() * sizeof(float),
              cudaMemcpyHostToDevice)) != cudaSuccess)) {
        delete p;
        return cuda_status(e, "Parker weight table");
    }
    if (p->tc_filter) {
        // Toeplitz operand T[j][k] = h(j-k) split into BF16 parts, each the
        // rounding of what the previous parts leave of h (FP64)
        const size_t tn = static_cast<size_t>(nu) * p->lda;
        const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
        std::vector<__nv_bfloat16> t0(tn, zero), t1(tn, zero), t2(p->tc_parts == 3 ? tn : 0, zero);
        for (int j = 0; j < nu; ++j)
            for (int k = 0; k < nu; ++k) {
                const size_t at = static_cast<size_t>(j) * p->lda + k;
                double v = h[static_cast<size_t>(j - k + nu - 1)];
                const __nv_bfloat16 b0 = __float2bfloat16_rn(static_cast<float>(v));
                v -= static_cast<double>(__bfloat162float(b0));
                const __nv_bfloat16 b1 = __float2bfloat16_rn(static_cast<float>(v));
                t0[at] = b0;
                t1[at] = b1;
                if (p->tc_parts == 3)
                    t2[at] = __float2bfloat16_rn(static_cast<float>(v - static_cast<double>(__bfloat162float(b1))));
            }
        p->tc_near = tc_filter_near_chunks(h, nu);
        if (const char* v = std::getenv("YKB_FDK_FILTER_NEAR"))
            if (std::atoi(v) > 0) p->tc_near = std::atoi(v);
        if ((e = p->toeplitz_hi.alloc(tn * 2)) != cudaSuccess ||
            (e = p->toeplitz_lo.alloc(tn * 2)) != cudaSuccess ||
            (p->tc_parts == 3 && (e = p->toeplitz_lo2.alloc(tn * 2)) != cudaSuccess) ||
            (e = cudaMemcpy(p->toeplitz_hi.ptr, t0.data(), tn * 2, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(p->toeplitz_lo.ptr, t1.data(), tn * 2, cudaMemcpyHostToDevice)) != cudaSuccess ||
            (p->tc_parts == 3 &&
             (e = cudaMemcpy(p->toeplitz_lo2.ptr, t2.data(), tn * 2, cudaMemcpyHostToDevice)) != cudaSuccess)) {
            delete p;
            return cuda_status(e, "Toeplitz operand");
        }
    }
    // size the shared-memory projection box of the TMA backprojection from
    // the footprints of every (tile, view) pair
    if (fdk_tma_available()) {
        cudaStream_t s = nullptr;
        if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) {
            delete p;
            return cuda_status(e, "cudaStreamCreate");
        }
        e = fdk_tma_box(p->coef.as<FdkViewCoef>(), n_views, make_grid(p->volume),
            p->err_flag.as<int>() + 2, &p->tma_bw, &p->tma_bh, s);
        cudaStreamDestroy(s);
        if (e != cudaSuccess) {
            delete p;
            return cuda_status(e, "backprojection box pre-pass");
        }
        p->use_tma = p->tma_bw > 0 && fdk_tma_stages(p->tma_bw, p->tma_bh, kFilteredScalar) > 0;
    }
    // YKB_FDK_BP_PATH=rows|global selects the plain-row TMA or the global-load
    // backprojection instead of the default (tests compare the three paths)
    const char* path = std::getenv("YKB_FDK_BP_PATH");
    const bool force_rows = path && std::strcmp(path, "rows") == 0;
    if (path && std::strcmp(path, "global") == 0) p->use_tma = false;
    // filtered workspace: tap pairs when their box fits the shared-memory
    // ring, else plain rows; both with 16-byte row pitch (TMA)
    p->layout = p->use_tma && !force_rows &&
        fdk_tma_stages(p->tma_bw, p->tma_bh, kFilteredPairs) > 0 ? kFilteredPairs : kFilteredScalar;
    p->ld = p->layout == kFilteredPairs ? (nu + kPairLead + 1) / 2 * 2 : (nu + 7) / 8 * 8;
    const size_t filt_bytes = static_cast<size_t>(p->batch_capacity) * p->ld * nv *
        (p->layout == kFilteredPairs ? 8 : 4);
    if ((e = p->work_filtered.alloc(filt_bytes)) != cudaSuccess) {
        delete p;
        return cuda_status(e, "cudaMalloc (FDK filtered workspace)");
    }
    *plan_out = p;
    return YKB_OK;
}

YKB_API ykb_status ykb_fdk_plan_destroy(ykb_fdk_plan* plan)
{
    clear_error();
    if (!plan) return YKB_OK;
    DeviceGuard guard(plan->device);
    delete plan;
    return YKB_OK;
}

YKB_API size_t ykb_fdk_workspace_bytes(const ykb_fdk_plan* p)
{
    if (!p) return 0;
    return p->coef.bytes + p->pwv.bytes + p->ramp.bytes + p->toeplitz_hi.bytes +
        p->toeplitz_lo.bytes + p->toeplitz_lo2.bytes + p->work_a.bytes + p->work_filtered.bytes +
        p->err_flag.bytes +
        p->parker.bytes + p->stage_in.bytes;
}

namespace {

ykb_status check_range(const ykb_fdk_plan* p, const void* buf, int dtype, int view_offset,
    int n_views)
{
    if (!p) return fail(YKB_ERR_INVALID_CONFIG, "null plan");
    if (!buf) return fail(YKB_ERR_INVALID_BUFFER, "null projection buffer");
    if (dtype != YKB_DTYPE_F32 && dtype != YKB_DTYPE_BF16)
        return fail(YKB_ERR_INVALID_CONFIG, "unknown projection dtype");
    if (view_offset < 0 || n_views <= 0 || view_offset > p->n_views - n_views)
        return fail(YKB_ERR_INVALID_CONFIG, "view_offset/n_views outside the prepared views");
    return YKB_OK;
}

size_t dtype_bytes(int dtype) { return dtype == YKB_DTYPE_BF16 ? 2 : 4; }

// Stage timing: the index of the event pair recorded around a stage's launch
// group, or -1 when the plan does not time its stages (or its pool of 4096
// pairs is full until the next ykb_fdk_stage_times)
int stage_begin(ykb_fdk_plan* p, int stage, cudaStream_t s)
{
    if (!p->timing || p->stage_events_used >= 4096) return -1;
    if (p->stage_events_used == p->stage_events.size()) {
        ykb_fdk_plan::StageEvents e;
        if (cudaEventCreate(&e.start) != cudaSuccess || cudaEventCreate(&e.stop) != cudaSuccess) {
            if (e.start) cudaEventDestroy(e.start);
            cudaGetLastError();
            return -1;
        }
        p->stage_events.push_back(e);
    }
    ykb_fdk_plan::StageEvents& e = p->stage_events[p->stage_events_used];
    e.stage = stage;
    if (cudaEventRecord(e.start, s) != cudaSuccess) return -1;
    return static_cast<int>(p->stage_events_used++);
}

void stage_end(ykb_fdk_plan* p, int i, cudaStream_t s)
{
    if (i >= 0) cudaEventRecord(p->stage_events[static_cast<size_t>(i)].stop, s);
}

// preweight + ramp for views [first, first+count) of the plan, input rows at
// proj, output into dst (FilteredLayout `layout`, row pitch ldc elements)
ykb_status filter_chunk_(ykb_fdk_plan* p, const void* proj, int proj_dtype, int first, int count,
    float* dst, int layout, int ldc, cudaStream_t s)
{
    const FdkPreweightView* pwv = p->pwv.as<FdkPreweightView>() + first;
    const float* parker = p->parker.ptr ? p->parker.as<float>() + static_cast<size_t>(first) * p->nu
                                        : nullptr;
    if (p->tc_filter) {
        const size_t part = static_cast<size_t>(p->batch_capacity) * p->nv * p->lda;
        __nv_bfloat16* a0 = p->work_a.as<__nv_bfloat16>();
        const __nv_bfloat16* const t[3] = {p->toeplitz_hi.as<__nv_bfloat16>(),
            p->toeplitz_lo.as<__nv_bfloat16>(),
            p->tc_parts == 3 ? p->toeplitz_lo2.as<__nv_bfloat16>() : nullptr};
        // sub-batches of views: the preweight (memory bound) of sub-batch
        // b + 1 runs on the auxiliary stream under the ramp filter (tensor
        // bound) of sub-batch b
        constexpr int kSub = ykb_fdk_plan::kFilterSubBatches;
        const int nsub = count >= 16 * kSub ? kSub : 1;
        if (nsub > 1 && !p->aux_stream) {
            YKB_TRY_CUDA(cudaStreamCreateWithFlags(&p->aux_stream, cudaStreamNonBlocking));
            YKB_TRY_CUDA(cudaEventCreateWithFlags(&p->aux_in, cudaEventDisableTiming));
            for (cudaEvent_t& e : p->aux_done)
                YKB_TRY_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        const cudaStream_t pw_stream = nsub > 1 ? p->aux_stream : s;
        if (nsub > 1) {
            // the input is ready and the previous filter call has read the parts
            YKB_TRY_CUDA(cudaEventRecord(p->aux_in, s));
            YKB_TRY_CUDA(cudaStreamWaitEvent(p->aux_stream, p->aux_in, 0));
        }
        const size_t in_esz = proj_dtype == YKB_DTYPE_BF16 ? 2 : 4;
        for (int b = 0; b < nsub; ++b) {
            const int v0 = static_cast<int>(static_cast<long>(count) * b / nsub);
            const int v1 = static_cast<int>(static_cast<long>(count) * (b + 1) / nsub);
            const size_t row0 = static_cast<size_t>(v0) * p->nv;
            __nv_bfloat16* const a[3] = {a0 + row0 * p->lda, a0 + part + row0 * p->lda,
                p->tc_parts == 3 ? a0 + 2 * part + row0 * p->lda : nullptr};
            YKB_TRY_CUDA(launch_fdk_preweight_split_bf16(
                static_cast<const char*>(proj) + row0 * p->nu * in_esz, proj_dtype, pwv + v0,
                parker ? parker + static_cast<size_t>(v0) * p->nu : nullptr, v1 - v0, p->nu, p->nv,
                p->lda, a, pw_stream));
            if (nsub > 1) YKB_TRY_CUDA(cudaEventRecord(p->aux_done[b], p->aux_stream));
        }
        for (int b = 0; b < nsub; ++b) {
            const int v0 = static_cast<int>(static_cast<long>(count) * b / nsub);
            const int v1 = static_cast<int>(static_cast<long>(count) * (b + 1) / nsub);
            const size_t row0 = static_cast<size_t>(v0) * p->nv;
            const __nv_bfloat16* const ac[3] = {a0 + row0 * p->lda, a0 + part + row0 * p->lda,
                p->tc_parts == 3 ? a0 + 2 * part + row0 * p->lda : nullptr};
            if (nsub > 1) YKB_TRY_CUDA(cudaStreamWaitEvent(s, p->aux_done[b], 0));
            const size_t out_row = layout == kFilteredPairs ? 2 * static_cast<size_t>(ldc)
                                                            : static_cast<size_t>(ldc);
            YKB_TRY_CUDA(launch_fdk_ramp_tcgen05(ac, t, (v1 - v0) * p->nv, p->nu, p->lda, pwv + v0,
                p->nv, dst + row0 * out_row, layout, ldc, p->tc_near, p->err_flag.as<int>(), s));
        }
        return YKB_OK;
    }
    YKB_TRY_CUDA(launch_fdk_preweight(proj, proj_dtype, pwv, parker, count, p->nu, p->nv,
        p->work_a.as<float>(), s));
    YKB_TRY_CUDA(launch_fdk_ramp_fp32(p->work_a.as<float>(), p->ramp.as<float>(), pwv, count,
        p->nu, p->nv, dst, layout, ldc, s));
    return YKB_OK;
}

ykb_status filter_chunk(ykb_fdk_plan* p, const void* proj, int proj_dtype, int first, int count,
    float* dst, int layout, int ldc, cudaStream_t s)
{
    const int ev = stage_begin(p, 0, s);
    const ykb_status st = filter_chunk_(p, proj, proj_dtype, first, count, dst, layout, ldc, s);
    stage_end(p, ev, s);
    return st;
}

// weighted backprojection of `count` filtered views (FilteredLayout
// `layout`, row pitch ld elements) starting at plan view `first`
// z_begin/z_count restrict the work to volume slices [z_begin, z_begin +
// z_count) (z_count < 0: all); z_begin must be a multiple of fdk_tma_z_tile()
// of the TMA backprojection, so that its tiles are those of the box pre-pass
ykb_status backproject_chunk_(ykb_fdk_plan* p, const void* filtered, int layout, int ld, int first,
    int count, float* vol, int accumulate, cudaStream_t s, int z_begin, int z_count)
{
    VolumeGrid grid = make_grid(p->volume);
    if (z_count >= 0) {
        vol += static_cast<size_t>(z_begin) * grid.nx * grid.ny;
        grid.oz += z_begin * grid.vz;
        grid.nz = z_count;
    }
    const FdkViewCoef* coef = p->coef.as<FdkViewCoef>() + first;
    const bool aligned = (reinterpret_cast<uintptr_t>(filtered) & 15) == 0;
    if (layout == kFilteredPairs) {
        YKB_TRY_CUDA(launch_fdk_backproject_tma(static_cast<const float*>(filtered), layout, ld,
            count, coef, count, p->nu, p->nv, grid, p->axial, p->tma_bw, p->tma_bh, vol,
            accumulate, p->err_flag.as<int>(), s, nullptr, p->bp_wait));
    } else if (p->use_tma && ld % 4 == 0 && aligned) {
        YKB_TRY_CUDA(launch_fdk_backproject_tma(static_cast<const float*>(filtered), layout, ld,
            count, coef, count, p->nu, p->nv, grid, p->axial, p->tma_bw, p->tma_bh, vol,
            accumulate, p->err_flag.as<int>(), s, nullptr, p->bp_wait));
    } else {
        YKB_TRY_CUDA(launch_fdk_backproject(filtered, YKB_DTYPE_F32, coef, count, p->nu, p->nv,
            ld, grid, p->axial, vol, accumulate, s));
    }
    return YKB_OK;
}

ykb_status backproject_chunk(ykb_fdk_plan* p, const void* filtered, int layout, int ld, int first,
    int count, float* vol, int accumulate, cudaStream_t s, int z_begin = 0, int z_count = -1)
{
    const int ev = stage_begin(p, 1, s);
    const ykb_status st = backproject_chunk_(p, filtered, layout, ld, first, count, vol,
        accumulate, s, z_begin, z_count);
    stage_end(p, ev, s);
    return st;
}

// Host projections streamed through the plan, copied on the plan's copy
// stream into two staging slots double-buffered against the filter and
// backprojection on `s`.  Batches double from 16 views up to half of the
// views: the kernels wait only for the first, short copy, and each later
// copy (a view copies in about half the time its kernels take) completes
// while the previous batch is processed; a remainder of between one and two
// batches runs as two halves.  Few batches matter: each backprojection
// launch costs about 0.8 ms beyond its views (512^3 x 720: 64.6 ms in one
// launch, 75.7 ms in seven).  With h_volume, the last batch is
// backprojected in z slabs of whole z tiles, about a quarter of the volume
// each (two 64-slice layers of 512 CTAs at 512^3 fill whole waves of 148
// SMs, where one layer leaves half a wave idle), and each finished slab is
// copied to h_volume behind the next slab's kernel; `s` then completes with
// the host volume.
ykb_status stream_host(ykb_fdk_plan* p, const void* h_proj, int proj_dtype, int view_offset,
    int n_views, float* d_volume, float* h_volume, int clear_output, cudaStream_t s)
{
    const size_t view_bytes = static_cast<size_t>(p->nu) * p->nv * dtype_bytes(proj_dtype);
    const int batch = std::min(p->batch_capacity, std::max(16, (p->n_views + 1) / 2));
    if (p->stage_views < batch || p->stage_in.bytes < 2 * batch * static_cast<size_t>(p->nu) * p->nv * 4) {
        if (p->copy_stream) YKB_TRY_CUDA(cudaStreamSynchronize(p->copy_stream));
        YKB_TRY_CUDA(cudaStreamSynchronize(s));
        YKB_TRY_CUDA(p->stage_in.alloc(2 * static_cast<size_t>(batch) * p->nu * p->nv * 4));
        p->stage_views = batch;
    }
    if (!p->copy_stream) {
        YKB_TRY_CUDA(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
        for (int i = 0; i < 2; ++i) {
            YKB_TRY_CUDA(cudaEventCreateWithFlags(&p->copied[i], cudaEventDisableTiming));
            YKB_TRY_CUDA(cudaEventCreateWithFlags(&p->consumed[i], cudaEventDisableTiming));
        }
    }
    // the copy stream starts after work already queued on `s` that may
    // still read the staging slots (a previous call)
    YKB_TRY_CUDA(cudaEventRecord(p->consumed[0], s));
    YKB_TRY_CUDA(cudaEventRecord(p->consumed[1], s));
    const size_t slot_bytes = static_cast<size_t>(p->stage_views) * view_bytes;
    int next_batch = std::min(batch, 16);
    const int nz = p->volume.nz;
    // quarters of the volume in whole z tiles: the download of the last slab
    // is what stays exposed
    const int zt = fdk_tma_z_tile();
    const int slab = std::max(zt, (nz / 4 + zt - 1) / zt * zt);
    const size_t plane = static_cast<size_t>(p->volume.nx) * p->volume.ny;
    for (int c = 0, b = 0; c < n_views; ++b) {
        // between one and two batches left: two halves, so that the last
        // batch, whose slabs hide the volume download, is never a short tail
        const int rest = n_views - c;
        const int cnt = rest > next_batch && rest < 2 * next_batch ? (rest + 1) / 2
                                                                  : std::min(next_batch, rest);
        next_batch = std::min(batch, 2 * next_batch);
        const int slot = b & 1;
        char* dst = static_cast<char*>(p->stage_in.ptr) + slot * slot_bytes;
        YKB_TRY_CUDA(cudaStreamWaitEvent(p->copy_stream, p->consumed[slot], 0));
        YKB_TRY_CUDA(cudaMemcpyAsync(dst, static_cast<const char*>(h_proj) + c * view_bytes,
            cnt * view_bytes, cudaMemcpyHostToDevice, p->copy_stream));
        YKB_TRY_CUDA(cudaEventRecord(p->copied[slot], p->copy_stream));
        YKB_TRY_CUDA(cudaStreamWaitEvent(s, p->copied[slot], 0));
        if (const ykb_status st = filter_chunk(p, dst, proj_dtype, view_offset + c, cnt,
                p->work_filtered.as<float>(), p->layout, p->ld, s))
            return st;
        YKB_TRY_CUDA(cudaEventRecord(p->consumed[slot], s));
        const int accumulate = (c == 0 && clear_output) ? 0 : 1;
        const bool last = c + cnt >= n_views;
        if (!last || !h_volume) {
            if (const ykb_status st = backproject_chunk(p, p->work_filtered.ptr, p->layout, p->ld,
                    view_offset + c, cnt, d_volume, accumulate, s))
                return st;
        } else {
            for (int z0 = 0, k = 0; z0 < nz; z0 += slab, ++k) {
                const int zc = std::min(slab, nz - z0);
                if (const ykb_status st = backproject_chunk(p, p->work_filtered.ptr, p->layout,
                        p->ld, view_offset + c, cnt, d_volume, accumulate, s, z0, zc))
                    return st;
                // slab k is final: the copy stream downloads it behind the
                // next slab's kernel (each wait binds to the record just made)
                cudaEvent_t done = p->copied[k & 1];
                YKB_TRY_CUDA(cudaEventRecord(done, s));
                YKB_TRY_CUDA(cudaStreamWaitEvent(p->copy_stream, done, 0));
                YKB_TRY_CUDA(cudaMemcpyAsync(h_volume + z0 * plane, d_volume + z0 * plane,
                    zc * plane * sizeof(float), cudaMemcpyDeviceToHost, p->copy_stream));
            }
            // the caller's stream completes when the host volume is complete
            YKB_TRY_CUDA(cudaEventRecord(p->consumed[0], p->copy_stream));
            YKB_TRY_CUDA(cudaStreamWaitEvent(s, p->consumed[0], 0));
        }
        c += cnt;
    }
    return YKB_OK;
}

} // namespace

YKB_API ykb_status ykb_fdk_filter(ykb_fdk_plan* p, const void* d_proj, int proj_dtype,
    int view_offset, int n_views, void* d_filtered, ykb_stream stream)
{
    clear_error();
    if (const ykb_status st = check_range(p, d_proj, proj_dtype, view_offset, n_views)) return st;
    if (!d_filtered) return fail(YKB_ERR_INVALID_BUFFER, "null filtered output");
    DeviceGuard guard(p->device);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t view_elems = static_cast<size_t>(p->nu) * p->nv;
    const size_t out_b = sizeof(float);
    for (int c = 0; c < n_views; c += p->batch_capacity) {
        const int cnt = std::min(p->batch_capacity, n_views - c);
        const char* in = static_cast<const char*>(d_proj) + c * view_elems * dtype_bytes(proj_dtype);
        float* out = reinterpret_cast<float*>(static_cast<char*>(d_filtered) + c * view_elems * out_b);
        if (const ykb_status st = filter_chunk(p, in, proj_dtype, view_offset + c, cnt, out,
                kFilteredScalar, p->nu, s))
            return st;
    }
    return YKB_OK;
}

YKB_API ykb_status ykb_fdk_backproject(ykb_fdk_plan* p, const void* d_filtered,
    int filtered_dtype, int view_offset, int n_views, float* d_volume, int clear_output,
    ykb_stream stream)
{
    clear_error();
    if (const ykb_status st = check_range(p, d_filtered, filtered_dtype, view_offset, n_views))
        return st;
    if (!d_volume) return fail(YKB_ERR_INVALID_BUFFER, "null volume buffer");
    DeviceGuard guard(p->device);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (filtered_dtype == YKB_DTYPE_BF16) {
        YKB_TRY_CUDA(launch_fdk_backproject(d_filtered, YKB_DTYPE_BF16,
            p->coef.as<FdkViewCoef>() + view_offset, n_views, p->nu, p->nv, p->nu,
            make_grid(p->volume), p->axial, d_volume, clear_output ? 0 : 1, s));
        return YKB_OK;
    }
    if (p->layout != kFilteredPairs)
        return backproject_chunk(p, d_filtered, kFilteredScalar, p->nu, view_offset, n_views,
            d_volume, clear_output ? 0 : 1, s);
    // plain rows from the caller: re-laid as tap pairs in the plan workspace
    const size_t view_elems = static_cast<size_t>(p->nu) * p->nv;
    for (int c = 0; c < n_views; c += p->batch_capacity) {
        const int cnt = std::min(p->batch_capacity, n_views - c);
        YKB_TRY_CUDA(launch_fdk_pairify(static_cast<const float*>(d_filtered) + c * view_elems,
            p->nu, static_cast<long>(cnt) * p->nv, p->nu, p->work_filtered.as<float>(), p->ld, s));
        const int accumulate = (c == 0 && clear_output) ? 0 : 1;
        if (const ykb_status st = backproject_chunk(p, p->work_filtered.ptr, kFilteredPairs, p->ld,
                view_offset + c, cnt, d_volume, accumulate, s))
            return st;
    }
    return YKB_OK;
}

YKB_API ykb_status ykb_fdk_execute(ykb_fdk_plan* p, const void* d_proj, int proj_dtype,
    int view_offset, int n_views, float* d_volume, int clear_output, ykb_stream stream)
{
    clear_error();
    if (const ykb_status st = check_range(p, d_proj, proj_dtype, view_offset, n_views)) return st;
    if (!d_volume) return fail(YKB_ERR_INVALID_BUFFER, "null volume buffer");
    DeviceGuard guard(p->device);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t view_elems = static_cast<size_t>(p->nu) * p->nv;
    for (int c = 0; c < n_views; c += p->batch_capacity) {
        const int cnt = std::min(p->batch_capacity, n_views - c);
        const char* in = static_cast<const char*>(d_proj) + c * view_elems * dtype_bytes(proj_dtype);
        if (const ykb_status st = filter_chunk(p, in, proj_dtype, view_offset + c, cnt,
                p->work_filtered.as<float>(), p->layout, p->ld, s))
            return st;
        const int accumulate = (c == 0 && clear_output) ? 0 : 1;
        if (const ykb_status st = backproject_chunk(p, p->work_filtered.ptr, p->layout, p->ld,
                view_offset + c, cnt, d_volume, accumulate, s))
            return st;
    }
    return YKB_OK;
}

YKB_API ykb_status ykb_fdk_execute_host(ykb_fdk_plan* p, const void* h_proj, int proj_dtype,
    int view_offset, int n_views, float* d_volume, int clear_output, ykb_stream stream)
{
    clear_error();
    if (const ykb_status st = check_range(p, h_proj, proj_dtype, view_offset, n_views)) return st;
    if (!d_volume) return fail(YKB_ERR_INVALID_BUFFER, "null volume buffer");
    DeviceGuard guard(p->device);
    return stream_host(p, h_proj, proj_dtype, view_offset, n_views, d_volume, nullptr,
        clear_output, reinterpret_cast<cudaStream_t>(stream));
}

YKB_API ykb_status ykb_fdk_execute_host_out(ykb_fdk_plan* p, const void* h_proj, int proj_dtype,
    int view_offset, int n_views, float* d_volume, float* h_volume, int clear_output,
    ykb_stream stream)
{
    clear_error();
    if (const ykb_status st = check_range(p, h_proj, proj_dtype, view_offset, n_views)) return st;
    if (!d_volume || !h_volume) return fail(YKB_ERR_INVALID_BUFFER, "null volume buffer");
    DeviceGuard guard(p->device);
    return stream_host(p, h_proj, proj_dtype, view_offset, n_views, d_volume, h_volume,
        clear_output, reinterpret_cast<cudaStream_t>(stream));
}

YKB_API ykb_status ykb_fdk_stage_timing(ykb_fdk_plan* p, int enable)
{
    clear_error();
    if (!p) return fail(YKB_ERR_INVALID_BUFFER, "null plan");
    p->timing = enable != 0;
    p->stage_events_used = 0;
    return YKB_OK;
}

YKB_API ykb_status ykb_fdk_stage_times(ykb_fdk_plan* p, ykb_stream stream, double* filter_ms,
    int* filter_groups, double* backproject_ms, int* backproject_groups)
{
    clear_error();
    if (!p || !filter_ms || !filter_groups || !backproject_ms || !backproject_groups)
        return fail(YKB_ERR_INVALID_BUFFER, "null plan or output");
    DeviceGuard guard(p->device);
    YKB_TRY_CUDA(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)));
    double ms[2] = {0.0, 0.0};
    int groups[2] = {0, 0};
    for (size_t i = 0; i < p->stage_events_used; ++i) {
        const auto& e = p->stage_events[i];
        YKB_TRY_CUDA(cudaEventSynchronize(e.stop));
        float t = 0.f;
        YKB_TRY_CUDA(cudaEventElapsedTime(&t, e.start, e.stop));
        ms[e.stage] += t;
        ++groups[e.stage];
    }
    p->stage_events_used = 0;
    *filter_ms = ms[0];
    *filter_groups = groups[0];
    *backproject_ms = ms[1];
    *backproject_groups = groups[1];
    return YKB_OK;
}

YKB_API ykb_status ykb_fdk_test_pipeline_wait(ykb_fdk_plan* p, unsigned long long wait_ns,
    int withheld_view)
{
    clear_error();
    if (!p) return fail(YKB_ERR_INVALID_BUFFER, "null plan");
    if (withheld_view < -1) return fail(YKB_ERR_INVALID_CONFIG, "withheld_view must be >= -1");
    p->bp_wait.limit_ns = wait_ns ? wait_ns : PipelineWait{}.limit_ns;
    p->bp_wait.withheld_view = withheld_view;
    return YKB_OK;
}

YKB_API ykb_status ykb_fdk_check(ykb_fdk_plan* p, ykb_stream stream)
{
    clear_error();
    if (!p) return fail(YKB_ERR_INVALID_CONFIG, "null plan");
    DeviceGuard guard(p->device);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int word = 0;
    YKB_TRY_CUDA(cudaMemcpyAsync(&word, p->err_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    YKB_TRY_CUDA(cudaStreamSynchronize(s));
    if (word == 0) return YKB_OK;
    YKB_TRY_CUDA(cudaMemsetAsync(p->err_flag.ptr, 0, sizeof(int), s));
    YKB_TRY_CUDA(cudaStreamSynchronize(s));
    std::string msg = "device-side failure in the backprojection:";
    if (word & 1) msg += " a pipeline wait timed out;";
    if (word & 2) msg += " a voxel column left its projection box;";
    if (word & 4) msg += " a staged copy was not 128-byte aligned (skipped);";
    if (word & 8) msg += " a tensor-core filter pipeline wait timed out;";
    return fail(YKB_ERR_CUDA, msg);
}

// --------------------------------------------------------------- Joseph ---
YKB_API ykb_status ykb_joseph_plan_create(const ykb_cone_view* views, int n_views, int nu, int nv,
    const ykb_volume* volume, int device, ykb_joseph_plan** plan_out)
{
    clear_error();
    if (!plan_out) return fail(YKB_ERR_INVALID_BUFFER, "null plan output");
    *plan_out = nullptr;
    if (!views || n_views <= 0 || nu <= 0 || nv <= 0)
        return fail(YKB_ERR_INVALID_CONFIG, "views, view count and detector size must be positive");
    if (!valid_volume(volume)) return fail(YKB_ERR_INVALID_CONFIG, "invalid volume grid");
    if (const ykb_status st = check_device(device)) return st;
    DeviceGuard guard(device);
    ykb_joseph_plan* p = new (std::nothrow) ykb_joseph_plan();
    if (!p) return fail(YKB_ERR_OUT_OF_MEMORY, "host allocation failed");
    p->device = device; p->n_views = n_views; p->nu = nu; p->nv = nv; p->volume = *volume;
    std::string why;
    p->cone_views.assign(views, views + n_views);
    if (!build_joseph_views(views, n_views, nu, nv, *volume, p->host_views, why)) {
        delete p;
        return fail(YKB_ERR_INVALID_GEOMETRY, why);
    }
    p->axes.resize(n_views);
    bool need_x = false, need_y = false;
    std::vector<float> vp(static_cast<size_t>(n_views) * 12);
    for (int i = 0; i < n_views; ++i) {
        const JosephView& j = p->host_views[i];
        p->axes[i] = j.axis;
        need_x |= j.axis == 0;
        need_y |= j.axis == 1;
        // voxel-space 3x4 projection (u w, v w, w) = M (x', y', z', 1)
        const double* S = j.src; const double* D0 = j.detS; const double* U = j.detU; const double* V = j.detV;
        const double n[3] = {U[1] * V[2] - U[2] * V[1], U[2] * V[0] - U[0] * V[2], U[0] * V[1] - U[1] * V[0]};
        auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
        const double sd[3] = {S[0] - D0[0], S[1] - D0[1], S[2] - D0[2]};
        const double plane = -dot(n, sd);
        const double W[4] = {n[0], n[1], n[2], -dot(n, S)};
        const double au = dot(sd, U), av = dot(sd, V);
        double DU[4], DV[4];
        for (int k = 0; k < 3; ++k) {
            DU[k] = au * W[k] + plane * U[k];
            DV[k] = av * W[k] + plane * V[k];
        }
        DU[3] = au * W[3] - plane * dot(U, S);
        DV[3] = av * W[3] - plane * dot(V, S);
        const double UU = dot(U, U), VV = dot(V, V), UV = dot(U, V);
        const double gram = UU * VV - UV * UV;
        if (!(std::fabs(gram) > 1e-30) || !(std::fabs(W[3]) > 1e-12)) {
            delete p;
            return fail(YKB_ERR_INVALID_GEOMETRY, "degenerate detector basis or source at the volume centre");
        }
        const double inv = 1.0 / gram, norm = 1.0 / W[3];
        for (int k = 0; k < 4; ++k) {
            vp[i * 12 + k] = static_cast<float>((DU[k] * VV - DV[k] * UV) * inv * norm);
            vp[i * 12 + 4 + k] = static_cast<float>((-DU[k] * UV + DV[k] * UU) * inv * norm);
            vp[i * 12 + 8 + k] = static_cast<float>(W[k] * norm);
        }
    }
    const size_t rays = static_cast<size_t>(n_views) * nu * nv;
    cudaError_t e;
    if ((e = p->views.alloc(sizeof(JosephView) * n_views)) != cudaSuccess ||
        (e = p->view_proj.alloc(sizeof(float) * vp.size())) != cudaSuccess ||
        (e = p->rays.alloc(sizeof(float4) * rays)) != cudaSuccess ||
        (e = p->lens.alloc(sizeof(float) * rays)) != cudaSuccess ||
        (need_y && (e = p->slab_y.alloc(sizeof(float) * joseph_slab_elems(*volume, 1))) != cudaSuccess) ||
        (need_x && (e = p->slab_x.alloc(sizeof(float) * joseph_slab_elems(*volume, 0))) != cudaSuccess)) {
        delete p;
        return cuda_status(e, "cudaMalloc (Joseph plan)");
    }
    if ((e = cudaMemcpy(p->views.ptr, p->host_views.data(), sizeof(JosephView) * n_views,
             cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(p->view_proj.ptr, vp.data(), sizeof(float) * vp.size(),
             cudaMemcpyHostToDevice)) != cudaSuccess) {
        delete p;
        return cuda_status(e, "cudaMemcpy (Joseph plan tables)");
    }
    // geometry-only ray table, built once on a private stream
    cudaStream_t s = nullptr;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) {
        delete p;
        return cuda_status(e, "cudaStreamCreate");
    }
    // the slabs' zero borders, written once (the transposes fill the interior)
    if (p->slab_y.ptr) e = cudaMemsetAsync(p->slab_y.ptr, 0, p->slab_y.bytes, s);
    if (e == cudaSuccess && p->slab_x.ptr) e = cudaMemsetAsync(p->slab_x.ptr, 0, p->slab_x.bytes, s);
    if (e == cudaSuccess)
        e = launch_joseph_ray_table(p->views.as<JosephView>(), n_views, nu, nv,
            p->rays.as<float4>(), p->lens.as<float>(), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    // the line backprojector when every view's main axis is x or y and its
    // detector columns are axial (YKB_JOSEPH_BP=gather keeps the gather)
    bool columns = std::none_of(p->axes.begin(), p->axes.end(), [](int a) { return a == 2; });
    if (const char* env = std::getenv("YKB_JOSEPH_BP"))
        if (std::strcmp(env, "gather") == 0) columns = false;
    if (e == cudaSuccess && columns) {
        DeviceBuffer flag;
        int differs = 1;
        if ((e = p->cols.alloc(sizeof(float2) * n_views * nu)) == cudaSuccess &&
            (e = flag.alloc(sizeof(int))) == cudaSuccess &&
            (e = launch_joseph_column_table(p->rays.as<float4>(), n_views, nu, nv,
                 p->cols.as<float2>(), flag.as<int>(), s)) == cudaSuccess &&
            (e = cudaMemcpyAsync(&differs, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s)) ==
                cudaSuccess)
            e = cudaStreamSynchronize(s);
        p->column_bp = e == cudaSuccess && differs == 0;
        if (!p->column_bp) p->cols.reset();
    }
    if (e == cudaSuccess)
        e = p->weighted.alloc(sizeof(float) * rays);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) {
        delete p;
        return cuda_status(e, "Joseph ray table");
    }
    *plan_out = p;
    return YKB_OK;
}

YKB_API ykb_status ykb_joseph_plan_destroy(ykb_joseph_plan* plan)
{
    clear_error();
    if (!plan) return YKB_OK;
    DeviceGuard guard(plan->device);
    delete plan;
    return YKB_OK;
}

YKB_API size_t ykb_joseph_workspace_bytes(const ykb_joseph_plan* p)
{
    if (!p) return 0;
    return p->views.bytes + p->view_proj.bytes + p->rays.bytes + p->lens.bytes +
        p->weighted.bytes + p->cols.bytes + p->slab_x.bytes + p->slab_y.bytes +
        p->world_views.bytes +
        p->fdk_coef.bytes +
        p->pseudo_coef.bytes + p->pairs.bytes + p->err_flag.bytes;
}

YKB_API ykb_status ykb_joseph_fp(ykb_joseph_plan* p, const float* d_volume, float* d_proj,
    int accumulate, ykb_stream stream)
{
    clear_error();
    if (!p) return fail(YKB_ERR_INVALID_CONFIG, "null plan");
    if (!d_volume || !d_proj) return fail(YKB_ERR_INVALID_BUFFER, "null volume or projection buffer");
    DeviceGuard guard(p->device);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const ykb_volume& v = p->volume;
    YKB_TRY_CUDA(launch_joseph_transpose(d_volume, v.nx, v.ny, v.nz, p->slab_y.as<float>(),
        p->slab_x.as<float>(), s));
    const float* slabs[3] = {p->slab_x.as<float>(), p->slab_y.as<float>(), d_volume};
    YKB_TRY_CUDA(launch_joseph_fp(slabs, p->views.as<JosephView>(), p->axes.data(), p->n_views,
        p->nu, p->nv, d_proj, accumulate ? 1 : 0, s));
    return YKB_OK;
}

} // extern "C"

namespace {

// Per-view tables of the pseudo-matched backprojection, built on first use:
// the FDK projection coefficients of the views (the reference derives them
// with the same GeoDerivedManagerVec for its operator, YkProjectionOperators.hpp:
// 249-251), the weight coefficients, and the TMA projection box.
ykb_status prepare_pseudo(ykb_joseph_plan* p, cudaStream_t s)
{
    if (p->pseudo_ready) return YKB_OK;
    std::vector<FdkDerived> g;
    std::string why;
    // the scan range only scales the FDK view weight, which this weight does not use
    if (!derive_fdk_geometry(p->cone_views.data(), p->n_views, p->nu, p->nv,
            6.28318530717958647692f, g, why))
        return fail(YKB_ERR_INVALID_GEOMETRY, why);
    std::vector<FdkViewCoef> coef;
    std::vector<FdkPreweightView> pw;
    bool axial = false;
    build_fdk_coefficients(g, p->nu, coef, pw, axial);
    p->pseudo_axial = axial;
    std::vector<PseudoViewCoef> pc;
    build_pseudo_coefficients(g, p->volume, pc);
    cudaError_t e;
    if ((e = p->fdk_coef.alloc(sizeof(FdkViewCoef) * coef.size())) != cudaSuccess ||
        (e = p->pseudo_coef.alloc(sizeof(PseudoViewCoef) * pc.size())) != cudaSuccess ||
        (e = p->err_flag.alloc(4 * sizeof(int))) != cudaSuccess)
        return cuda_status(e, "cudaMalloc (pseudo-matched tables)");
    YKB_TRY_CUDA(cudaMemcpyAsync(p->fdk_coef.ptr, coef.data(), p->fdk_coef.bytes,
        cudaMemcpyHostToDevice, s));
    YKB_TRY_CUDA(cudaMemcpyAsync(p->pseudo_coef.ptr, pc.data(), p->pseudo_coef.bytes,
        cudaMemcpyHostToDevice, s));
    YKB_TRY_CUDA(cudaMemsetAsync(p->err_flag.ptr, 0, p->err_flag.bytes, s));
    p->pseudo_bw = p->pseudo_bh = 0;
    if (fdk_tma_available() && !std::getenv("YKB_PSEUDO_BP_GLOBAL")) {
        int bw = 0, bh = 0;
        YKB_TRY_CUDA(fdk_tma_box(p->fdk_coef.as<FdkViewCoef>(), p->n_views,
            make_grid(p->volume), p->err_flag.as<int>() + 2, &bw, &bh, s));
        if (bw > 0 && fdk_tma_stages(bw, bh, kFilteredPairs) > 0) {
            const int ld = (p->nu + kPairLead + 1) / 2 * 2;
            if (p->pairs.alloc(static_cast<size_t>(p->n_views) * p->nv * ld * 8) == cudaSuccess) {
                p->pseudo_bw = bw;
                p->pseudo_bh = bh;
                p->pseudo_ld = ld;
            } else {
                // without room for the staged pairs the bounds-checked kernel runs
                cudaGetLastError();
            }
        }
    }
    YKB_TRY_CUDA(cudaStreamSynchronize(s));
    p->pseudo_ready = true;
    return YKB_OK;
}

ykb_status pseudo_bp(ykb_joseph_plan* p, const float* d_proj, float* d_volume, int accumulate,
    cudaStream_t s)
{
    if (const ykb_status st = prepare_pseudo(p, s)) return st;
    const VolumeGrid g = make_grid(p->volume);
    if (p->pseudo_bw > 0) {
        YKB_TRY_CUDA(launch_fdk_pairify(d_proj, p->nu, static_cast<long>(p->n_views) * p->nv,
            p->nu, p->pairs.as<float>(), p->pseudo_ld, s));
        YKB_TRY_CUDA(launch_fdk_backproject_tma(p->pairs.as<float>(), kFilteredPairs,
            p->pseudo_ld, p->n_views, p->fdk_coef.as<FdkViewCoef>(), p->n_views, p->nu, p->nv, g,
            p->pseudo_axial, p->pseudo_bw, p->pseudo_bh, d_volume, accumulate,
            p->err_flag.as<int>(), s,
            p->pseudo_coef.as<PseudoViewCoef>()));
        return YKB_OK;
    }
    YKB_TRY_CUDA(launch_pseudo_backproject(d_proj, p->fdk_coef.as<FdkViewCoef>(),
        p->pseudo_coef.as<PseudoViewCoef>(), p->n_views, p->nu, p->nv, g, d_volume, accumulate, s));
    return YKB_OK;
}

ykb_status siddon(ykb_joseph_plan* p, bool forward, const float* d_in, float* d_out,
    int accumulate, cudaStream_t s)
{
    if (!p->world_views.ptr) {
        const size_t bytes = sizeof(ykb_cone_view) * p->cone_views.size();
        cudaError_t e = p->world_views.alloc(bytes);
        if (e != cudaSuccess) return cuda_status(e, "cudaMalloc (Siddon views)");
        e = cudaMemcpyAsync(p->world_views.ptr, p->cone_views.data(), bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            p->world_views.reset();
            return cuda_status(e, "cudaMemcpy (Siddon views)");
        }
    }
    const VolumeGrid g = make_grid(p->volume);
    const ykb_cone_view* v = p->world_views.as<ykb_cone_view>();
    if (forward)
        YKB_TRY_CUDA(launch_siddon_fp(d_in, v, p->n_views, p->nu, p->nv, g, d_out, accumulate, s));
    else
        YKB_TRY_CUDA(launch_siddon_bp(d_in, v, p->n_views, p->nu, p->nv, g, d_out, accumulate, s));
    return YKB_OK;
}

} // namespace

extern "C" {

YKB_API ykb_status ykb_operator_apply(ykb_joseph_plan* p, int task, const float* d_in,
    float* d_out, int accumulate, ykb_stream stream)
{
    clear_error();
    if (!p) return fail(YKB_ERR_INVALID_CONFIG, "null plan");
    switch (task) {
    case YKB_TASK_FP_JOSEPH: return ykb_joseph_fp(p, d_in, d_out, accumulate, stream);
    case YKB_TASK_BP_JOSEPH: return ykb_joseph_bp(p, d_in, d_out, accumulate, stream);
    case YKB_TASK_FP_SIDDON:
    case YKB_TASK_BP_SIDDON_RAY_DRIVEN: {
        if (!d_in || !d_out) return fail(YKB_ERR_INVALID_BUFFER, "null volume or projection buffer");
        DeviceGuard guard(p->device);
        return siddon(p, task == YKB_TASK_FP_SIDDON, d_in, d_out, accumulate ? 1 : 0,
            reinterpret_cast<cudaStream_t>(stream));
    }
    case YKB_TASK_BP_FDK_PSEUDO_MATCHED: {
        if (!d_in || !d_out) return fail(YKB_ERR_INVALID_BUFFER, "null volume or projection buffer");
        DeviceGuard guard(p->device);
        return pseudo_bp(p, d_in, d_out, accumulate ? 1 : 0, reinterpret_cast<cudaStream_t>(stream));
    }
    default:
        return fail(YKB_ERR_UNSUPPORTED, "operator task " + std::to_string(task) + " is not implemented");
    }
}

YKB_API ykb_status ykb_joseph_check(ykb_joseph_plan* p, ykb_stream stream)
{
    clear_error();
    if (!p) return fail(YKB_ERR_INVALID_CONFIG, "null plan");
    if (!p->err_flag.ptr) return YKB_OK;
    DeviceGuard guard(p->device);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int word = 0;
    YKB_TRY_CUDA(cudaMemcpyAsync(&word, p->err_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    YKB_TRY_CUDA(cudaStreamSynchronize(s));
    if (word == 0) return YKB_OK;
    YKB_TRY_CUDA(cudaMemsetAsync(p->err_flag.ptr, 0, sizeof(int), s));
    YKB_TRY_CUDA(cudaStreamSynchronize(s));
    std::string msg = "device-side failure in the pseudo-matched backprojection:";
    if (word & 1) msg += " a pipeline wait timed out;";
    if (word & 2) msg += " a voxel column left its projection box;";
    if (word & 4) msg += " a staged copy was not 128-byte aligned (skipped);";
    return fail(YKB_ERR_CUDA, msg);
}

// ------------------------------------------------- iterative solvers ---
YKB_API ykb_status ykb_iter_create(int device, ykb_iter** ctx)
{
    clear_error();
    if (!ctx) return fail(YKB_ERR_INVALID_BUFFER, "null context output");
    *ctx = nullptr;
    if (const ykb_status st = check_device(device)) return st;
    DeviceGuard guard(device);
    ykb_iter* c = new (std::nothrow) ykb_iter();
    if (!c) return fail(YKB_ERR_OUT_OF_MEMORY, "host allocation failed");
    c->device = device;
    const cudaError_t e = c->partials.alloc(sizeof(double) * dot_partial_count());
    if (e != cudaSuccess) {
        delete c;
        return cuda_status(e, "cudaMalloc (reduction workspace)");
    }
    *ctx = c;
    return YKB_OK;
}

YKB_API ykb_status ykb_iter_destroy(ykb_iter* ctx)
{
    clear_error();
    if (!ctx) return YKB_OK;
    DeviceGuard guard(ctx->device);
    delete ctx;
    return YKB_OK;
}

YKB_API ykb_status ykb_dot_f64(ykb_iter* ctx, const float* d_a, const float* d_b, size_t n,
    double* d_result, ykb_stream stream)
{
    clear_error();
    if (!ctx) return fail(YKB_ERR_INVALID_CONFIG, "null context");
    if (!d_result || (n > 0 && (!d_a || !d_b))) return fail(YKB_ERR_INVALID_BUFFER, "null buffer");
    DeviceGuard guard(ctx->device);
    YKB_TRY_CUDA(launch_dot_f64(d_a, d_b, n, ctx->partials.as<double>(), d_result,
        reinterpret_cast<cudaStream_t>(stream)));
    return YKB_OK;
}

YKB_API ykb_status ykb_cgls_update_xr(ykb_iter* ctx, const double* d_gamma, const double* d_ww,
    float* d_x, const float* d_p, size_t nx, float* d_r, const float* d_w, size_t nr,
    ykb_stream stream)
{
    clear_error();
    if (!ctx) return fail(YKB_ERR_INVALID_CONFIG, "null context");
    if (!d_gamma || !d_ww || !d_x || !d_p || !d_r || !d_w) return fail(YKB_ERR_INVALID_BUFFER, "null buffer");
    DeviceGuard guard(ctx->device);
    YKB_TRY_CUDA(launch_cgls_xr(d_gamma, d_ww, d_x, d_p, nx, d_r, d_w, nr,
        reinterpret_cast<cudaStream_t>(stream)));
    return YKB_OK;
}

YKB_API ykb_status ykb_cgls_update_p(ykb_iter* ctx, const double* d_gamma_new,
    const double* d_gamma_old, float* d_p, const float* d_z, size_t n, ykb_stream stream)
{
    clear_error();
    if (!ctx) return fail(YKB_ERR_INVALID_CONFIG, "null context");
    if (!d_gamma_new || !d_gamma_old || !d_p || !d_z) return fail(YKB_ERR_INVALID_BUFFER, "null buffer");
    DeviceGuard guard(ctx->device);
    YKB_TRY_CUDA(launch_cgls_p(d_gamma_new, d_gamma_old, d_p, d_z, n,
        reinterpret_cast<cudaStream_t>(stream)));
    return YKB_OK;
}

YKB_API ykb_status ykb_joseph_bp(ykb_joseph_plan* p, const float* d_proj, float* d_volume,
    int accumulate, ykb_stream stream)
{
    clear_error();
    if (!p) return fail(YKB_ERR_INVALID_CONFIG, "null plan");
    if (!d_volume || !d_proj) return fail(YKB_ERR_INVALID_BUFFER, "null volume or projection buffer");
    DeviceGuard guard(p->device);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (p->column_bp)
        YKB_TRY_CUDA(launch_joseph_bp_lines(d_proj, p->rays.as<float4>(), p->lens.as<float>(),
            p->cols.as<float2>(), p->view_proj.as<float>(), p->views.as<JosephView>(),
            p->n_views, p->nu, p->nv, p->volume, p->weighted.as<float>(), d_volume,
            accumulate ? 1 : 0, s));
    else
        YKB_TRY_CUDA(launch_joseph_bp(d_proj, p->rays.as<float4>(), p->lens.as<float>(),
            p->view_proj.as<float>(), p->views.as<JosephView>(), p->n_views, p->nu, p->nv,
            p->volume, p->weighted.as<float>(), d_volume, accumulate ? 1 : 0, s));
    return YKB_OK;
}

} // extern "C"
