// ykb_fdk_filter_static: the FDK preweight + ramp filter stage without any
// device allocation.  Its scratch (ramp lags, per-view preweight records and
// the preweighted rows between the two kernels) lives in one file-scope
// device array of fixed size; the caller passes only inputs and outputs.
//
// For callers that cannot call cudaMalloc: processes that hand all GPU
// memory to their own pool at start-up, real-time acquisition loops that
// forbid allocation after initialisation, and code running while another
// component owns the allocator.
#include "ykb_internal.hpp"

#include <algorithm>
#include <mutex>

namespace ykb {
namespace {

// 32 MiB per device, held by every GPU that loads the library until exit:
// 64 KiB of ramp lags, 2.5 MiB of per-view records and 30,867,456 bytes
// (29.4 MiB) for the preweighted rows of the views filtered at once.
constexpr size_t kStaticBytes = size_t(32) << 20;
constexpr int kStaticMaxNu = 8192;       // ramp lags: 2*nu-1 floats
constexpr int kStaticMaxViews = 16384;   // per-view records
constexpr size_t kLagBytes = sizeof(float) * (2 * kStaticMaxNu);
constexpr size_t kRecordBytes = sizeof(FdkPreweightView) * kStaticMaxViews;
constexpr size_t kRowsOffset = ((kLagBytes + kRecordBytes + 255) / 256) * 256;
constexpr size_t kRowsBytes = kStaticBytes - kRowsOffset;

static __device__ __align__(256) unsigned char g_filter_scratch[kStaticBytes];

// The symbol names a host-side stand-in, not a device address: each device's
// address is looked up once, with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

ykb_status scratch_for_device(int device, unsigned char** out)
{
    if (device < 0 || device >= kMaxDevices)
        return (set_error("device index outside the static scratch table"), YKB_ERR_INVALID_CONFIG);
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_filter_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_filter_scratch)");
        g_scratch_ptr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[device]);
    return YKB_OK;
}

} // namespace
} // namespace ykb

using namespace ykb;

extern "C" YKB_API ykb_status ykb_fdk_filter_static(const ykb_cone_view* views, int n_views,
    int nu, int nv, float scan_range_rad, const ykb_filter* filter, const void* d_proj,
    int proj_dtype, float* d_filtered, ykb_stream stream)
{
    clear_error();
    if (!views || n_views <= 0 || nu <= 0 || nv <= 0 || !filter)
        return (set_error("views, filter, view count and detector size are required"),
            YKB_ERR_INVALID_CONFIG);
    if (!d_proj || !d_filtered)
        return (set_error("null projection or filtered buffer"), YKB_ERR_INVALID_BUFFER);
    if (proj_dtype != YKB_DTYPE_F32 && proj_dtype != YKB_DTYPE_BF16)
        return (set_error("unknown projection dtype"), YKB_ERR_INVALID_CONFIG);
    if (filter->type < 0 || filter->type > 9 || !(filter->cutoff > 0.f) || filter->cutoff > 0.5f ||
        !(filter->gain > 0.f) || !(filter->butterworth_order > 0.f) || filter->kaiser_beta < 0.f ||
        filter->tukey_alpha < 0.f || filter->tukey_alpha > 1.f)
        return (set_error("invalid analytic filter parameters"), YKB_ERR_INVALID_CONFIG);
    const size_t view_bytes = sizeof(float) * static_cast<size_t>(nu) * nv;
    if (nu > kStaticMaxNu || n_views > kStaticMaxViews || view_bytes > kRowsBytes)
        return (set_error("ykb_fdk_filter_static limits: nu <= 8192, n_views <= 16384 and one "
                          "view's nu*nv*4 bytes <= " + std::to_string(kRowsBytes) + " bytes"),
            YKB_ERR_INVALID_CONFIG);
    // a short scan needs Parker redundancy weights between the preweight and
    // the filter, which take the scan's start angle and direction: a plan
    // (ykb_fdk_plan_create_ex) applies them; this entry point has no such
    // arguments and refuses rather than return unweighted rows
    if (scan_range_rad < 6.28318530717958647692f - 1e-5f)
        return (set_error("ykb_fdk_filter_static filters full scans only (scan range >= 2 pi): "
                          "a short scan needs Parker weights, which a plan from "
                          "ykb_fdk_plan_create_ex applies"), YKB_ERR_INVALID_CONFIG);
    int device = 0;
    if (const cudaError_t e = cudaGetDevice(&device)) return cuda_status(e, "cudaGetDevice");
    unsigned char* base = nullptr;
    if (const ykb_status st = scratch_for_device(device, &base)) return st;

    std::vector<FdkDerived> derived;
    std::string why;
    if (!derive_fdk_geometry(views, n_views, nu, nv, scan_range_rad, derived, why))
        return (set_error(why), YKB_ERR_INVALID_GEOMETRY);
    std::vector<FdkViewCoef> coef;
    std::vector<FdkPreweightView> pw;
    bool axial = false;
    build_fdk_coefficients(derived, nu, coef, pw, axial);
    std::vector<double> h;
    build_ramp_kernel(nu, derived[0].du, *filter, h);
    std::vector<float> hf(h.begin(), h.end());

    float* d_lags = reinterpret_cast<float*>(base);
    FdkPreweightView* d_records = reinterpret_cast<FdkPreweightView*>(base + kLagBytes);
    float* d_rows = reinterpret_cast<float*>(base + kRowsOffset);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // every scratch byte read below is written first on the same stream:
    // the lags and records by these copies, the rows by the preweight kernel
    YKB_TRY_CUDA(cudaMemcpyAsync(d_lags, hf.data(), sizeof(float) * hf.size(),
        cudaMemcpyHostToDevice, s));
    YKB_TRY_CUDA(cudaMemcpyAsync(d_records, pw.data(), sizeof(FdkPreweightView) * n_views,
        cudaMemcpyHostToDevice, s));
    const int chunk = static_cast<int>(std::min<size_t>(n_views, kRowsBytes / view_bytes));
    const size_t in_elem = proj_dtype == YKB_DTYPE_BF16 ? 2 : 4;
    for (int c = 0; c < n_views; c += chunk) {
        const int cnt = std::min(chunk, n_views - c);
        const char* in = static_cast<const char*>(d_proj) +
            static_cast<size_t>(c) * nu * nv * in_elem;
        YKB_TRY_CUDA(launch_fdk_preweight(in, proj_dtype, d_records + c, nullptr, cnt, nu, nv,
            d_rows, s));
        YKB_TRY_CUDA(launch_fdk_ramp_fp32(d_rows, d_lags, d_records + c, cnt, nu, nv,
            d_filtered + static_cast<size_t>(c) * nu * nv, kFilteredScalar, nu, s));
    }
    // the host-side tables were copied from pageable memory: the copies have
    // left the host buffers when cudaMemcpyAsync returns
    return YKB_OK;
}
