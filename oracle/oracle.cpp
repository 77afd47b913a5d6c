// FP64 CPU oracle for YKCBCT's flat-panel circular FDK and Joseph FP/BP.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py as the checker.  The product library never
// links or calls this file.  Citations are paths inside the reference
// repository (YuuKozlx/fdk_cuda_impl).

#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr float kTwoPiF = 6.28318530717958647692f;

// ---------------------------------------------------------------------------
// float vector helpers used by the float geometry builders
// ---------------------------------------------------------------------------
struct f3 { float x, y, z; };
inline f3 mk(float x, float y, float z) { return {x, y, z}; }
inline float dotf(const f3& a, const f3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline f3 crossf(const f3& a, const f3& b)
{ return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline f3 addf(const f3& a, const f3& b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline f3 subf(const f3& a, const f3& b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline f3 scalef(const f3& v, float s) { return mk(v.x * s, v.y * s, v.z * s); }
inline f3 normf(const f3& v)
{
    const float l2 = dotf(v, v);
    if (!(l2 > 0.f)) return mk(0.f, 0.f, 0.f);
    return scalef(v, 1.f / std::sqrt(l2));
}
// Rodrigues rotation, include/YKCBCT/geometry/YkDetectorGeometryBuilders.hpp:37-44
inline f3 rot_axis(const f3& value, const f3& axis, float angle)
{
    const f3 unit = normf(axis);
    const float c = std::cos(angle), s = std::sin(angle);
    return addf(addf(scalef(value, c), scalef(crossf(unit, value), s)),
        scalef(unit, dotf(unit, value) * (1.f - c)));
}
// include/YKCBCT/geometry/YkTrajectoryGeometryBuilder.hpp:11-16
inline f3 rot_z(const f3& v, float angle)
{
    const float c = std::cos(angle), s = std::sin(angle);
    return mk(c * v.x - s * v.y, s * v.x + c * v.y, v.z);
}

// ---------------------------------------------------------------------------
// double vector helpers
// ---------------------------------------------------------------------------
struct d3 { double x, y, z; };
inline d3 md(double x, double y, double z) { return {x, y, z}; }
inline d3 d_of(const float* v) { return md(v[0], v[1], v[2]); }
inline double dotd(const d3& a, const d3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline d3 crossd(const d3& a, const d3& b)
{ return md(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline d3 addd(const d3& a, const d3& b) { return md(a.x + b.x, a.y + b.y, a.z + b.z); }
inline d3 subd(const d3& a, const d3& b) { return md(a.x - b.x, a.y - b.y, a.z - b.z); }
inline d3 scaled(const d3& v, double s) { return md(v.x * s, v.y * s, v.z * s); }
inline double lend(const d3& v) { return std::sqrt(dotd(v, v)); }

// ---------------------------------------------------------------------------
// Derived FDK geometry in FP64, restating
// src/Reconstruction/Analytic/Circular/Flat/FDK/YkFDKVecGeoDerived.hpp:58-304
// and include/YKCBCT/geometry/YkProjectionGeometry.hpp:114-194.
// ---------------------------------------------------------------------------
struct Derived {
    double theta, dtheta, fscale;
    double sid;            // source_to_axis_mm
    double dsd;            // source_to_radial_detector_mm
    double plane;          // source_to_detector_plane_mm
    double off_u, off_v;   // principal point offsets, pixels
    double du, dv;
    d3 src, detS, detU, detV, n, radial;
    double UU, VV, UV, inv_gram;
    int startU;
    bool ok;
};

// fp_computePaddedN, .../FDK/kernels/YkFDKFilterHelpers.cuh:29-34
int padded_n(int nu)
{
    int n = 1;
    while (n < 2 * nu) n <<= 1;
    return n;
}

// fp_computeStartU, .../FDK/kernels/YkFDKFilterHelpers.cuh:37-42 (float math
// on purpose: it is an integer placement decision taken in float).
int start_u(int nu, int padded, float offset_u)
{
    const float axis = (nu - 1) * 0.5f + offset_u;
    return static_cast<int>(lrintf(padded * 0.5f - axis));
}

bool derive(const orc_view* views, int n, int nu, int nv, float range,
    std::vector<Derived>& out)
{
    if (n <= 0 || nu <= 0 || nv <= 0 || !(range > 0.f)) return false;
    out.assign(n, Derived{});
    // theta unwrap (YkFDKVecGeoDerived.hpp:158-168) and central-difference
    // dtheta with eps 1e-8 (:173-184).  The angle inputs are floats; their
    // differences are exact in double.
    std::vector<double> th(n);
    for (int i = 0; i < n; ++i) th[i] = views[i].angle[0];
    for (int i = 1; i < n; ++i) {
        double t = th[i];
        const double p = th[i - 1];
        while (t - p > kPi) t -= 2 * kPi;
        while (t - p < -kPi) t += 2 * kPi;
        th[i] = t;
    }
    const int padded = padded_n(nu);
    for (int i = 0; i < n; ++i) {
        Derived& g = out[i];
        const orc_view& v = views[i];
        g.theta = th[i];
        double dt;
        if (n <= 1) dt = 1e-8;
        else if (i == 0) dt = th[1] - th[0];
        else if (i == n - 1) dt = th[n - 1] - th[n - 2];
        else dt = 0.5 * (th[i + 1] - th[i - 1]);
        dt = std::fabs(dt);
        if (dt < 1e-8) dt = 1e-8;
        g.dtheta = dt;
        g.fscale = 2.0 * kPi / static_cast<double>(range);
        g.src = d_of(v.src); g.detS = d_of(v.detS);
        g.detU = d_of(v.detU); g.detV = d_of(v.detV);
        g.du = lend(g.detU); g.dv = lend(g.detV);
        // deriveProjectionFrame: normal from detV x detU, oriented towards the
        // detector centre; plane distance (detS - src).n
        const d3 centre = addd(g.detS, addd(scaled(g.detU, 0.5 * (nu - 1)),
            scaled(g.detV, 0.5 * (nv - 1))));
        const d3 cdir = subd(centre, g.src);
        d3 nrm = crossd(g.detV, g.detU);
        const double nl = lend(nrm);
        if (!(nl > 1e-12) || !(lend(cdir) > 1e-12)) return false;
        nrm = scaled(nrm, 1.0 / nl);
        if (dotd(nrm, cdir) < 0) nrm = scaled(nrm, -1.0);
        g.n = nrm;
        g.plane = dotd(subd(g.detS, g.src), nrm);
        if (!(g.plane > 1e-12)) return false;
        // compute_radial_ray: source to the closest point on the z axis
        // through the origin (YkFDKVecGeoDerived.hpp:194-209)
        const d3 closest = md(0.0, 0.0, g.src.z);
        const d3 ray = subd(closest, g.src);
        const double rl = lend(ray);
        if (!(rl > 1e-10)) return false;
        g.sid = rl;
        g.radial = scaled(ray, 1.0 / rl);
        // compute_SDD_offsets (YkFDKVecGeoDerived.hpp:257-304)
        const double den = dotd(g.radial, nrm);
        if (std::fabs(den) < 1e-12) return false;
        const double t = g.plane / den;
        if (!(t > 0)) return false;
        const d3 pp = addd(g.src, scaled(g.radial, t));
        g.dsd = lend(subd(pp, g.src));
        g.UU = dotd(g.detU, g.detU);
        g.VV = dotd(g.detV, g.detV);
        g.UV = dotd(g.detU, g.detV);
        const double gram = g.UU * g.VV - g.UV * g.UV;
        if (std::fabs(gram) < 1e-20) return false;
        g.inv_gram = 1.0 / gram;
        const d3 D = subd(pp, g.detS);
        const double DU = dotd(D, g.detU), DV = dotd(D, g.detV);
        g.off_u = (DU * g.VV - DV * g.UV) * g.inv_gram - 0.5 * (nu - 1);
        g.off_v = (-DU * g.UV + DV * g.UU) * g.inv_gram - 0.5 * (nv - 1);
        g.startU = start_u(nu, padded, static_cast<float>(g.off_u));
        g.ok = true;
    }
    return true;
}

// Voxel-centre world coordinate, include/YKCBCT/geometry/YkVolumeGeometry.hpp:47-53
inline double vox_centre(int i, int n, float vox, float centre)
{
    return static_cast<double>(centre) + (i - 0.5 * (n - 1)) * static_cast<double>(vox);
}

// Projection of a world point on the detector of one view, in pixel units
// with pixel (0,0) at detS, by ray/plane intersection and the Gram solve
// (the direct form of .../FDK/kernels/YkFDKBpKernels.cu:63-104 with the
// non-orthogonal basis inversion of YkFDKBpPrecompute.cu:80-87).  Returns
// the radial depth (P-src).radial used by the FDK distance weight.
inline void project_point(const Derived& g, const d3& P, double& u, double& v,
    double& depth)
{
    const d3 dir = subd(P, g.src);
    depth = dotd(dir, g.radial);
    const double dn = dotd(dir, g.n);
    const double t = g.plane / dn;
    const d3 D = subd(addd(g.src, scaled(dir, t)), g.detS);
    const double DU = dotd(D, g.detU), DV = dotd(D, g.detV);
    u = (DU * g.VV - DV * g.UV) * g.inv_gram;
    v = (-DU * g.UV + DV * g.UU) * g.inv_gram;
}

// Emulation of the texture unit's linear filter, which the reference's FDK
// backprojection (tex2D) and Joseph projector (tex3D) read through: the
// fraction of the texel coordinate is held with 8 fractional bits (CUDA C
// Programming Guide, "Texture Fetching", linear filtering).  The rounding is
// to nearest with ties upward, alpha = floor(256 f + 0.5) / 256: measured on a
// B200 by fetching a ramp texture at 327680 coordinates, in 2D and 3D, which
// this rule reproduces exactly.
inline double tex_frac(double f) { return std::floor(f * 256.0 + 0.5) / 256.0; }

template <typename T>
inline double bilerp_zero(const T* img, int w, int h, double x, double y,
    bool tex_emulation)
{
    const double fx = std::floor(x), fy = std::floor(y);
    const long ix = static_cast<long>(fx), iy = static_cast<long>(fy);
    double ax = x - fx, ay = y - fy;
    if (tex_emulation) { ax = tex_frac(ax); ay = tex_frac(ay); }
    auto at = [&](long xx, long yy) -> double {
        if (xx < 0 || yy < 0 || xx >= w || yy >= h) return 0.0;
        return static_cast<double>(img[yy * static_cast<long>(w) + xx]);
    };
    return (1 - ay) * ((1 - ax) * at(ix, iy) + ax * at(ix + 1, iy)) +
        ay * ((1 - ax) * at(ix, iy + 1) + ax * at(ix + 1, iy + 1));
}

// ---------------------------------------------------------------------------
// Ramp filter weights.  AnalyticFreq construction of
// src/Filter/YkCreateFilterKernelKernels.cu:167-191 with the windows of
// src/Filter/YkCreateFilterKernelHelpers.cuh:38-103 and the 1/du scale of
// src/Filter/YkCreateFilterKernelFFT.hpp:181-190 (identity kind: :166-170).
// ---------------------------------------------------------------------------
double bessel_i0(double x)
{
    // power series sum_k ((x/2)^k / k!)^2
    const double q = 0.25 * x * x;
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 500; ++k) {
        term *= q / (static_cast<double>(k) * k);
        sum += term;
        if (term < 1e-17 * sum) break;
    }
    return sum;
}

double window_shape(double x, const orc_filter& f)
{
    x = std::min(std::max(x, 0.0), 1.0);
    switch (f.type) {
    case 1: return 1.0;
    case 2: { const double t = kPi * 0.5 * x;
        return std::fabs(t) < 1e-8 ? 1.0 : std::sin(t) / t; }
    case 3: return std::cos(0.5 * kPi * x);
    case 4: return 0.5 * (1.0 + std::cos(kPi * x));
    case 5: return 0.54 + 0.46 * std::cos(kPi * x);
    case 6: return 0.42 + 0.5 * std::cos(kPi * x) + 0.08 * std::cos(2.0 * kPi * x);
    case 7: { const double order = std::max(static_cast<double>(f.butterworth_order), 0.01);
        return 1.0 / (1.0 + std::pow(x, 2.0 * order)); }
    case 8: { const double beta = std::max(static_cast<double>(f.kaiser_beta), 0.0);
        const double t = 2.0 * x - 1.0;
        return bessel_i0(beta * std::sqrt(std::max(0.0, 1.0 - t * t))) / bessel_i0(beta); }
    case 9: { const double a = std::min(std::max(static_cast<double>(f.tukey_alpha), 0.0), 1.0);
        if (a <= 0.0) return 1.0;
        if (x < a * 0.5) return 0.5 * (1.0 + std::cos(kPi * (2.0 * x / a - 1.0)));
        if (x <= 1.0 - a * 0.5) return 1.0;
        return 0.5 * (1.0 + std::cos(kPi * (2.0 * x / a - 2.0 / a + 1.0))); }
    default: return 1.0;
    }
}

// Frequency weights w[k], k=0..N/2, with 1/N baked in.
void freq_weights(int N, double du, const orc_filter& f, std::vector<double>& w)
{
    const int nc = N / 2 + 1;
    w.assign(nc, 0.0);
    const double invN = 1.0 / N;
    if (f.type == 0) {
        for (int k = 0; k < nc; ++k) w[k] = static_cast<double>(f.gain) * invN;
        return;
    }
    const double cc = f.cutoff > 0.f ? static_cast<double>(f.cutoff) : 0.5;
    for (int k = 0; k < nc; ++k) {
        const double fr = static_cast<double>(k) / N;
        if (fr > cc) { w[k] = 0.0; continue; }
        w[k] = static_cast<double>(f.gain) * fr * window_shape(fr / cc, f) * invN / du;
    }
}

// Circular kernel h[n] = IDFT_N of the Hermitian extension of w, as the cuFFT
// C2R of .../FDK/kernels/YkFDKFilterKernels.cu:114-125 computes it, evaluated
// for lags d = -(nu-1)..(nu-1) (the padded length N >= 2nu makes the circular
// convolution on the placed samples a linear Toeplitz one).
void ramp_kernel(int nu, double du, const orc_filter& f, std::vector<double>& h)
{
    const int N = padded_n(nu);
    std::vector<double> w;
    freq_weights(N, du, f, w);
    h.assign(2 * nu - 1, 0.0);
    for (int d = -(nu - 1); d <= nu - 1; ++d) {
        double s = w[0];
        for (int k = 1; k < N / 2; ++k)
            s += 2.0 * w[k] * std::cos(2.0 * kPi * static_cast<double>(k) * d / N);
        s += w[N / 2] * ((d & 1) ? -1.0 : 1.0);
        h[d + nu - 1] = s;
    }
}

// ---------------------------------------------------------------------------
// Joseph geometry: normalizeToVoxel (src/common/cuda/operators/
// YkOperatorKernelTypes.cuh:148-168) and the float main-axis decision of
// forEachAxisRun/mainAxis (:133-141,179-210) on the float frame of
// deriveProjectionFrame (include/YKCBCT/geometry/YkProjectionGeometry.hpp:114-194).
// ---------------------------------------------------------------------------
int main_axis_float(const orc_view& v, int nu, int nv)
{
    const f3 s = mk(v.src[0], v.src[1], v.src[2]);
    const f3 ds = mk(v.detS[0], v.detS[1], v.detS[2]);
    const f3 du = mk(v.detU[0], v.detU[1], v.detU[2]);
    const f3 dv = mk(v.detV[0], v.detV[1], v.detV[2]);
    const float cu = 0.5f * static_cast<float>(nu - 1);
    const float cv = 0.5f * static_cast<float>(nv - 1);
    const f3 c = mk(ds.x + cu * du.x + cv * dv.x, ds.y + cu * du.y + cv * dv.y,
        ds.z + cu * du.z + cv * dv.z);
    const f3 d = mk(c.x - s.x, c.y - s.y, c.z - s.z);
    const float l2 = d.x * d.x + d.y * d.y + d.z * d.z;
    if (!std::isfinite(l2) || l2 <= 1e-12f) return -1;
    const float inv = 1.f / std::sqrt(l2);
    const float ax = std::fabs(d.x * inv), ay = std::fabs(d.y * inv), az = std::fabs(d.z * inv);
    if (ax >= ay && ax >= az) return 0;
    if (ay >= ax && ay >= az) return 1;
    return 2;
}

struct JosephView {
    int axis;          // 0 X, 1 Y, 2 Z
    d3 src, detS, detU, detV;   // voxel units, volume-centred
    int n0, n1, n2;
    double v0, v1, v2;
};

inline double comp(const d3& p, int axis, int which)
{
    // which 0 -> c0 (main), 1 -> c1, 2 -> c2 (AxisX/AxisY/AxisZ permutations)
    static const int map[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
    const int k = map[axis][which];
    return k == 0 ? p.x : (k == 1 ? p.y : p.z);
}

bool joseph_views(const orc_view* views, int n, int nu, int nv,
    const orc_volume& vol, std::vector<JosephView>& out)
{
    out.resize(n);
    const double ix = 1.0 / vol.vox_x, iy = 1.0 / vol.vox_y, iz = 1.0 / vol.vox_z;
    for (int i = 0; i < n; ++i) {
        const orc_view& v = views[i];
        JosephView& j = out[i];
        j.axis = main_axis_float(v, nu, nv);
        if (j.axis < 0) return false;
        auto pt = [&](const float* p) {
            return md((p[0] - static_cast<double>(vol.center_x)) * ix,
                (p[1] - static_cast<double>(vol.center_y)) * iy,
                (p[2] - static_cast<double>(vol.center_z)) * iz);
        };
        j.src = pt(v.src);
        j.detS = pt(v.detS);
        j.detU = md(v.detU[0] * ix, v.detU[1] * iy, v.detU[2] * iz);
        j.detV = md(v.detV[0] * ix, v.detV[1] * iy, v.detV[2] * iz);
        const int dims[3] = {vol.nx, vol.ny, vol.nz};
        const double vx[3] = {vol.vox_x, vol.vox_y, vol.vox_z};
        static const int map[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
        j.n0 = dims[map[j.axis][0]]; j.n1 = dims[map[j.axis][1]]; j.n2 = dims[map[j.axis][2]];
        j.v0 = vx[map[j.axis][0]]; j.v1 = vx[map[j.axis][1]]; j.v2 = vx[map[j.axis][2]];
    }
    return true;
}

// Ray parameters of fp_joseph_kernel (src/FlatFpBp/FP/kernels/YkFPKernels.cu:
// 158-187): slopes a1,a2, intercepts b1,b2 in volume-centred voxel units and
// the anisotropic chord length per main-axis step.
struct Ray { double a1, b1, a2, b2, len; bool ok; };

inline Ray ray_params(const JosephView& j, int iu, int iv)
{
    const d3 det = addd(j.detS, addd(scaled(j.detU, iu), scaled(j.detV, iv)));
    Ray r{};
    const double dc0 = comp(j.src, j.axis, 0) - comp(det, j.axis, 0);
    if (std::fabs(dc0) < 1e-12) { r.ok = false; return r; }
    r.a1 = (comp(j.src, j.axis, 1) - comp(det, j.axis, 1)) / dc0;
    r.a2 = (comp(j.src, j.axis, 2) - comp(det, j.axis, 2)) / dc0;
    r.b1 = comp(j.src, j.axis, 1) - r.a1 * comp(j.src, j.axis, 0);
    r.b2 = comp(j.src, j.axis, 2) - r.a2 * comp(j.src, j.axis, 0);
    const double a1v1 = r.a1 * j.v1, a2v2 = r.a2 * j.v2;
    r.len = std::sqrt(j.v0 * j.v0 + a1v1 * a1v1 + a2v2 * a2v2);
    r.ok = true;
    return r;
}

inline size_t vox_index(const orc_volume& vol, int axis, int s, int j1, int j2)
{
    int x, y, z;
    if (axis == 0) { x = s; y = j1; z = j2; }
    else if (axis == 1) { x = j1; y = s; z = j2; }
    else { x = j1; y = j2; z = s; }
    return (static_cast<size_t>(z) * vol.ny + y) * vol.nx + x;
}

bool valid_volume(const orc_volume* v)
{
    return v && v->nx > 0 && v->ny > 0 && v->nz > 0 && v->vox_x > 0.f &&
        v->vox_y > 0.f && v->vox_z > 0.f;
}

// ---------------------------------------------------------------------------
// Deterministic random streams: splitmix64-seeded mt19937_64 per block of
// 65536 elements, so the output is independent of the thread count.
// ---------------------------------------------------------------------------
inline uint64_t splitmix(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
inline double uni01(std::mt19937_64& g) { return (g() >> 11) * (1.0 / 9007199254740992.0); }

// Poisson sampler: Knuth's product method for small mean, PTRS
// (W. Hormann, "The transformed rejection method for generating Poisson
// random variables", Insurance: Math. & Econ. 12, 1993) for mean >= 10.
long poisson(std::mt19937_64& g, double mu)
{
    if (mu <= 0) return 0;
    if (mu < 10.0) {
        const double L = std::exp(-mu);
        long k = 0;
        double p = uni01(g);
        while (p > L) { ++k; p *= uni01(g); }
        return k;
    }
    const double slam = std::sqrt(mu), loglam = std::log(mu);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2);
    for (;;) {
        const double U = uni01(g) - 0.5;
        const double V = uni01(g);
        const double us = 0.5 - std::fabs(U);
        const double k = std::floor((2 * a / us + b) * U + mu + 0.43);
        if (us >= 0.07 && V <= vr) return static_cast<long>(k);
        if (k < 0 || (us < 0.013 && V > us)) continue;
        if (std::log(V) + std::log(invalpha) - std::log(a / (us * us) + b) <=
            -mu + k * loglam - std::lgamma(k + 1))
            return static_cast<long>(k);
    }
}

} // namespace

namespace {
template <typename F>
void siddon_ray(const orc_view& vw, int iu, int iv, const orc_volume& V, F&& f)
{
    const double S[3] = {vw.src[0], vw.src[1], vw.src[2]};
    double r[3], lo[3], vox[3];
    const int N[3] = {V.nx, V.ny, V.nz};
    const double c[3] = {V.center_x, V.center_y, V.center_z};
    vox[0] = V.vox_x; vox[1] = V.vox_y; vox[2] = V.vox_z;
    for (int a = 0; a < 3; ++a) {
        const double D = static_cast<double>(vw.detS[a]) + iu * static_cast<double>(vw.detU[a]) +
            iv * static_cast<double>(vw.detV[a]);
        r[a] = D - S[a];
        lo[a] = c[a] - 0.5 * (N[a] - 1) * vox[a] - 0.5 * vox[a];
    }
    const double len = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    double tmin = 0.0, tmax = 1.0;
    for (int a = 0; a < 3; ++a) {
        const double hi = lo[a] + N[a] * vox[a];
        if (std::fabs(r[a]) > 1e-8) {
            double ta = (lo[a] - S[a]) / r[a], tb = (hi - S[a]) / r[a];
            if (ta > tb) std::swap(ta, tb);
            tmin = std::max(tmin, ta);
            tmax = std::min(tmax, tb);
        } else if (S[a] < lo[a] || S[a] > hi) {
            return;
        }
    }
    if (!(tmin < tmax)) return;
    std::vector<double> ts{tmin, tmax};
    for (int a = 0; a < 3; ++a) {
        if (!(std::fabs(r[a]) > 1e-8)) continue;
        for (int k = 0; k <= N[a]; ++k) {
            const double t = (lo[a] + k * vox[a] - S[a]) / r[a];
            if (t > tmin && t < tmax) ts.push_back(t);
        }
    }
    std::sort(ts.begin(), ts.end());
    for (size_t q = 0; q + 1 < ts.size(); ++q) {
        const double t0 = ts[q], t1 = ts[q + 1];
        if (!(t1 > t0)) continue;
        const double tm = 0.5 * (t0 + t1);
        long idx[3];
        bool in = true;
        for (int a = 0; a < 3; ++a) {
            idx[a] = static_cast<long>(std::floor((S[a] + tm * r[a] - lo[a]) / vox[a]));
            in = in && idx[a] >= 0 && idx[a] < N[a];
        }
        if (in) f((idx[2] * V.ny + idx[1]) * V.nx + idx[0], (t1 - t0) * len);
    }
}
} // namespace

extern "C" {

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// include/YKCBCT/interface/YkSystemReconstruction.hpp:22-28
float orc_regular_scan_range(int total_views, int views_per_turn)
{
    return kTwoPiF * static_cast<float>(total_views) / static_cast<float>(views_per_turn);
}

// buildCircularTrajectory + buildScannerViewFramesImpl + buildFlatProjectionGeometry:
// include/YKCBCT/geometry/YkSystemGeometry.hpp:37-73,
// include/YKCBCT/geometry/YkTrajectoryGeometryBuilder.hpp:29-67,
// include/YKCBCT/geometry/YkDetectorGeometryBuilders.hpp:46-107.
int orc_build_circular_flat(const orc_circular_flat* sp, orc_view* out)
{
    if (!sp || !out) return -1;
    const orc_circular_flat& s = *sp;
    if (!(s.total_views > 0 && s.views_per_turn >= 2 &&
          (s.rotation_direction == 1 || s.rotation_direction == -1) &&
          s.sid_mm > 0.f && s.sdd_mm > s.sid_mm && std::isfinite(s.start_angle_rad) &&
          std::isfinite(s.z_mm)))
        return -2;
    if (s.channels <= 0 || s.rows <= 0 || !(s.channel_size_mm > 0.f) || !(s.row_size_mm > 0.f))
        return -3;
    const float step = static_cast<float>(s.rotation_direction) * kTwoPiF /
        static_cast<float>(s.views_per_turn);
    const float dd = s.sdd_mm - s.sid_mm;
    const float cu = 0.5f * (s.channels - 1);
    const float cv = 0.5f * (s.rows - 1);
    for (int i = 0; i < s.total_views; ++i) {
        const float angle = s.start_angle_rad + i * step;
        const f3 zs = mk(0.f, 0.f, s.z_mm);
        const f3 src_local = mk(s.source_offset_mm[0], -s.sid_mm + s.source_offset_mm[1],
            s.source_offset_mm[2]);
        const f3 det_local = mk(0.f, dd, 0.f);
        auto shifted = [&](const f3& v) {
            const f3 r = rot_z(v, angle);
            return mk(r.x + zs.x, r.y + zs.y, r.z + zs.z);
        };
        const f3 source = shifted(src_local);
        const f3 principal = shifted(det_local);
        f3 u = rot_z(mk(1.f, 0.f, 0.f), angle);
        f3 v = mk(0.f, 0.f, 1.f);
        f3 n = rot_z(mk(0.f, -1.f, 0.f), angle);
        v = rot_axis(v, u, s.tilt_u_rad);
        n = rot_axis(n, u, s.tilt_u_rad);
        u = rot_axis(u, v, s.tilt_v_rad);
        n = rot_axis(n, v, s.tilt_v_rad);
        u = rot_axis(u, n, s.tilt_n_rad);
        v = rot_axis(v, n, s.tilt_n_rad);
        u = normf(u);
        v = normf(v);
        n = normf(crossf(u, v));
        if (dotf(n, subf(source, principal)) < 0.f) n = scalef(n, -1.f);
        const f3 centre = addf(principal, addf(scalef(u, s.offset_unv_mm[0]),
            addf(scalef(n, s.offset_unv_mm[1]), scalef(v, s.offset_unv_mm[2]))));
        const f3 du = scalef(u, s.channel_size_mm);
        const f3 dv = scalef(v, s.row_size_mm);
        const f3 start = subf(subf(centre, scalef(du, cu)), scalef(dv, cv));
        orc_view& o = out[i];
        const float src4[4] = {source.x, source.y, source.z, 0.f};
        const float ds4[4] = {start.x, start.y, start.z, 0.f};
        const float du4[4] = {du.x, du.y, du.z, 0.f};
        const float dv4[4] = {dv.x, dv.y, dv.z, 0.f};
        const float an4[4] = {angle, 0.f, 0.f, 0.f};
        std::memcpy(o.src, src4, sizeof src4);
        std::memcpy(o.detS, ds4, sizeof ds4);
        std::memcpy(o.detU, du4, sizeof du4);
        std::memcpy(o.detV, dv4, sizeof dv4);
        std::memcpy(o.angle, an4, sizeof an4);
    }
    return 0;
}

int orc_fdk_derived(const orc_view* views, int n, int nu, int nv, float range,
    double* out)
{
    std::vector<Derived> g;
    if (!derive(views, n, nu, nv, range, g)) return -1;
    for (int i = 0; i < n; ++i) {
        double* o = out + 12 * i;
        o[0] = g[i].theta; o[1] = g[i].dtheta; o[2] = g[i].fscale;
        o[3] = g[i].sid; o[4] = g[i].dsd; o[5] = g[i].plane;
        o[6] = g[i].off_u; o[7] = g[i].off_v; o[8] = g[i].du; o[9] = g[i].dv;
        o[10] = g[i].startU; o[11] = 0.0;
    }
    return 0;
}

int orc_ramp_kernel(int nu, double du, const orc_filter* f, double* h)
{
    if (nu <= 0 || !(du > 0) || !f) return -1;
    std::vector<double> hv;
    ramp_kernel(nu, du, *f, hv);
    std::copy(hv.begin(), hv.end(), h);
    return 0;
}

// Parker short-scan weights, restating
// .../FDK/kernels/YkFDKParkerKernels.cu:46-110 (weight per column, sin^2 ramps
// of width 2(Gamma +- gamma)), pk_uploadAngles :117-138 (beta), the
// processor's scale range/pi (.../FDK/YkFDKParkerWeightProcessor.hpp:30-40)
// and the coverage check of YkFdkPipeline.hpp:597-635.
int orc_parker_weights(const orc_view* views, int n, int nu, int nv, float range,
    float start_angle, int direction, double* w)
{
    if (!views || !w || n <= 0 || nu <= 0 || nv <= 0 || (direction != 1 && direction != -1))
        return -1;
    std::vector<Derived> g;
    if (!derive(views, n, nu, nv, range, g)) return -2;
    const double pi = kPi;
    if (static_cast<double>(range) >= 2.0 * pi - 1e-5) return -3;
    const double cv = 0.5 * (nv - 1);
    // coverage: pi + 2 * the largest edge fan angle against the principal ray
    double max_fan = 0.0;
    for (int i = 0; i < n; ++i) {
        const Derived& d = g[i];
        const d3 c = addd(d.detS, addd(scaled(d.detU, 0.5 * (nu - 1)), scaled(d.detV, cv)));
        const double px = c.x - d.src.x, py = c.y - d.src.y;
        for (double u : {0.0, static_cast<double>(nu - 1)}) {
            const d3 e = addd(d.detS, addd(scaled(d.detU, u), scaled(d.detV, cv)));
            const double rx = e.x - d.src.x, ry = e.y - d.src.y;
            max_fan = std::max(max_fan, std::fabs(std::atan2(rx * py - ry * px, rx * px + ry * py)));
        }
    }
    if (static_cast<double>(range) + 1e-5 < pi + 2.0 * max_fan) return -3;
    const double scale = static_cast<double>(range) / pi;
    const double eps = 1e-6;
    for (int i = 0; i < n; ++i) {
        const Derived& d = g[i];
        auto fan = [&](double u) {
            const double rx = d.detS.x + u * d.detU.x + cv * d.detV.x - d.src.x;
            const double ry = d.detS.y + u * d.detU.y + cv * d.detV.y - d.src.y;
            return std::atan2(rx * d.radial.y - ry * d.radial.x, rx * d.radial.x + ry * d.radial.y);
        };
        const double Gamma = std::max(std::fabs(fan(0.0)), std::fabs(fan(nu - 1.0)));
        double beta = direction * (static_cast<double>(views[i].angle[0]) - start_angle);
        while (beta < 0.0) beta += 2.0 * pi;
        while (beta >= 2.0 * pi) beta -= 2.0 * pi;
        for (int u = 0; u < nu; ++u) {
            const double gamma = direction * fan(u);
            const double t1 = 2.0 * (Gamma + gamma), t2 = pi + 2.0 * gamma, t3 = pi + 2.0 * Gamma;
            double x;
            if (beta <= 0.0) {
                x = 0.0;
            } else if (beta < t1) {
                const double dd = Gamma + gamma;
                const double sn = std::sin(0.25 * pi * beta / (std::fabs(dd) > eps ? dd : eps));
                x = sn * sn;
            } else if (beta <= t2) {
                x = 1.0;
            } else if (beta < t3) {
                const double dd = Gamma - gamma;
                const double sn = std::sin(0.25 * pi * (t3 - beta) / (std::fabs(dd) > eps ? dd : eps));
                x = sn * sn;
            } else {
                x = 0.0;
            }
            w[static_cast<size_t>(i) * nu + u] = x * scale;
        }
    }
    return 0;
}

// Preweight (.../FDK/kernels/YkFDKPreWeightKernels.cu:374-402) followed by the
// padded circular convolution (.../FDK/kernels/YkFDKFilterKernels.cu:32-125),
// written as its equivalent masked Toeplitz product.
int orc_fdk_filter(const orc_view* views, int n, int nu, int nv, float range,
    const orc_filter* filter, const float* proj, double* filtered)
{
    return orc_fdk_filter_weighted(views, n, nu, nv, range, filter, proj, nullptr, filtered);
}

namespace {

// Rows [row0, row0 + nrows) of the preweighted and ramp-filtered
// projections (proj and filtered hold only those rows, [n][nrows][nu]).  The
// filter acts on each detector row alone, so a band of rows filters exactly
// as it would inside the full detector.
void filter_rows(const std::vector<Derived>& g, const std::vector<double>& h, int n, int nu,
    int row0, int nrows, const float* proj, const double* row_weights, double* filtered)
{
    const int N = padded_n(nu);
#pragma omp parallel
    {
        std::vector<double> row(nu);
#pragma omp for schedule(static)
        for (long r = 0; r < static_cast<long>(n) * nrows; ++r) {
            const int i = static_cast<int>(r / nrows);
            const int iv = row0 + static_cast<int>(r % nrows);
            const Derived& d = g[i];
            const double wgeom = d.dsd / d.sid / 2.0;
            const float* src = proj + static_cast<size_t>(r) * nu;
            for (int iu = 0; iu < nu; ++iu) {
                const d3 q = subd(addd(d.detS, addd(scaled(d.detU, iu), scaled(d.detV, iv))), d.src);
                const double wcos = d.dsd / std::sqrt(std::max(dotd(q, q), 1e-20));
                const bool placed = (iu + d.startU) >= 0 && (iu + d.startU) < N;
                const double extra = row_weights ? row_weights[static_cast<size_t>(i) * nu + iu] : 1.0;
                row[iu] = placed ? static_cast<double>(src[iu]) * wcos * wgeom * extra : 0.0;
            }
            double* dst = filtered + static_cast<size_t>(r) * nu;
            for (int j = 0; j < nu; ++j) {
                const bool valid = (j + d.startU) >= 0 && (j + d.startU) < N;
                double s = 0.0;
                if (valid)
                    for (int k = 0; k < nu; ++k) s += row[k] * h[j - k + nu - 1];
                dst[j] = s;
            }
        }
    }
}

// Voxel-driven weighted backprojection (.../FDK/kernels/YkFDKBpKernels.cu:
// 112-209 with the coefficient definitions of YkFDKBpPrecompute.cu:14-138):
// vol += sum_views bilinear(u,v) * SID^2 * dtheta * (2pi/range) / depth^2,
// bilinear with zero border at pixel coordinates (u,v).  The filtered rows
// present are [row0, row0 + nrows); rows outside read as zero.
void backproject_rows(const std::vector<Derived>& g, int n, int nu, int row0, int nrows,
    const orc_volume& V, const double* filtered, double* volume, bool tex)
{
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < V.nz; ++z)
        for (int y = 0; y < V.ny; ++y)
            for (int x = 0; x < V.nx; ++x) {
                const d3 P = md(vox_centre(x, V.nx, V.vox_x, V.center_x),
                    vox_centre(y, V.ny, V.vox_y, V.center_y),
                    vox_centre(z, V.nz, V.vox_z, V.center_z));
                double acc = 0.0;
                for (int i = 0; i < n; ++i) {
                    const Derived& d = g[i];
                    double u, v, depth;
                    project_point(d, P, u, v, depth);
                    const double w = d.sid * d.sid * d.dtheta * d.fscale / (depth * depth);
                    acc += w * bilerp_zero(filtered + static_cast<size_t>(i) * nu * nrows,
                        nu, nrows, u, v - row0, tex);
                }
                volume[(static_cast<size_t>(z) * V.ny + y) * V.nx + x] += acc;
            }
}

} // namespace

int orc_fdk_filter_weighted(const orc_view* views, int n, int nu, int nv, float range,
    const orc_filter* filter, const float* proj, const double* row_weights, double* filtered)
{
    if (!filter || !proj || !filtered) return -1;
    std::vector<Derived> g;
    if (!derive(views, n, nu, nv, range, g)) return -2;
    std::vector<double> h;
    // the reference builds the weights once, with du of the first view of the
    // first chunk (.../FDK/YkFDKFilterProcessor.hpp:111,216-232)
    ramp_kernel(nu, g[0].du, *filter, h);
    filter_rows(g, h, n, nu, 0, nv, proj, row_weights, filtered);
    return 0;
}

int orc_fdk_backproject(const orc_view* views, int n, int nu, int nv,
    float range, const orc_volume* vol, const double* filtered, double* volume,
    int flags)
{
    if (!valid_volume(vol) || !filtered || !volume) return -1;
    std::vector<Derived> g;
    if (!derive(views, n, nu, nv, range, g)) return -2;
    backproject_rows(g, n, nu, 0, nv, *vol, filtered, volume, (flags & 1) != 0);
    return 0;
}

int orc_fdk_row_band(const orc_view* views, int n, int nu, int nv, float range,
    const orc_volume* vol, int* row0, int* nrows)
{
    if (!valid_volume(vol) || !row0 || !nrows) return -1;
    std::vector<Derived> g;
    if (!derive(views, n, nu, nv, range, g)) return -2;
    const orc_volume& V = *vol;
    const double xs[2] = {vox_centre(0, V.nx, V.vox_x, V.center_x),
                          vox_centre(V.nx - 1, V.nx, V.vox_x, V.center_x)};
    const double ys[2] = {vox_centre(0, V.ny, V.vox_y, V.center_y),
                          vox_centre(V.ny - 1, V.ny, V.vox_y, V.center_y)};
    const double zs[2] = {vox_centre(0, V.nz, V.vox_z, V.center_z),
                          vox_centre(V.nz - 1, V.nz, V.vox_z, V.center_z)};
    double vmin = 1e300, vmax = -1e300;
    for (int i = 0; i < n; ++i)
        for (int q = 0; q < 8; ++q) {
            double u, v, depth;
            project_point(g[i], md(xs[q & 1], ys[(q >> 1) & 1], zs[q >> 2]), u, v, depth);
            if (!(depth > 0.0)) return -3;  // a corner behind the source
            vmin = std::min(vmin, v);
            vmax = std::max(vmax, v);
        }
    const long lo = std::max(0L, static_cast<long>(std::floor(vmin)) - 1);
    const long hi = std::min(static_cast<long>(nv) - 1, static_cast<long>(std::floor(vmax)) + 2);
    if (lo > hi) { *row0 = 0; *nrows = 0; return 0; }
    *row0 = static_cast<int>(lo);
    *nrows = static_cast<int>(hi - lo + 1);
    return 0;
}

int orc_fdk_rows(const orc_view* views, int n, int nu, int nv, int row0, int nrows,
    float range, const orc_volume* vol, const orc_filter* filter, const float* proj_rows,
    const double* row_weights, double* volume_out, int flags)
{
    if (!valid_volume(vol) || !filter || !proj_rows || !volume_out) return -1;
    if (row0 < 0 || nrows <= 0 || row0 + nrows > nv) return -1;
    std::vector<Derived> g;
    if (!derive(views, n, nu, nv, range, g)) return -2;
    std::vector<double> h;
    ramp_kernel(nu, g[0].du, *filter, h);
    std::vector<double> flt(static_cast<size_t>(n) * nu * nrows);
    filter_rows(g, h, n, nu, row0, nrows, proj_rows, row_weights, flt.data());
    std::fill(volume_out, volume_out + static_cast<size_t>(vol->nx) * vol->ny * vol->nz, 0.0);
    backproject_rows(g, n, nu, row0, nrows, *vol, flt.data(), volume_out, (flags & 1) != 0);
    return 0;
}

// Siddon pair: FP_Siddon (siddon_fp_tex_kernel with a Point/Border texture,
// src/FlatFpBp/FP/kernels/YkFPSiddonKernel.cu:129-234,283-316, applied by
// ForwardOperator::apply, src/common/YkProjectionOperators.hpp:159-171) and
// BP_Siddon_RayDriven (siddon_bp_kernel, src/FlatFpBp/BP/kernels/
// YkBPSiddonKernel.cu:31-127).  The ray S + t (D - S) from the source to the
// pixel centre D, t in [0, 1] clipped to the outer voxel faces, contributes
// vol[voxel] x (length of the ray inside the voxel) -- here computed by
// Siddon's original parametric method: every face crossing in the clipped
// range, sorted, each interval assigned to the voxel holding its midpoint.

int orc_siddon_fp(const orc_view* views, int n, int nu, int nv, const orc_volume* vol,
    const float* volume, double* proj)
{
    if (!valid_volume(vol) || !views || !volume || !proj) return -1;
    const orc_volume V = *vol;
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = 0; k < n; ++k)
        for (int iv = 0; iv < nv; ++iv)
            for (int iu = 0; iu < nu; ++iu) {
                double acc = 0.0;
                siddon_ray(views[k], iu, iv, V, [&](long i, double l) { acc += volume[i] * l; });
                proj[(static_cast<size_t>(k) * nv + iv) * nu + iu] = acc;
            }
    return 0;
}

int orc_siddon_bp(const orc_view* views, int n, int nu, int nv, const orc_volume* vol,
    const float* proj, double* volume)
{
    if (!valid_volume(vol) || !views || !volume || !proj) return -1;
    const orc_volume V = *vol;
    const size_t nvox = static_cast<size_t>(V.nx) * V.ny * V.nz;
    std::fill(volume, volume + nvox, 0.0);
    // per-thread partial volumes keep the sum deterministic
#pragma omp parallel
    {
        std::vector<double> part(nvox, 0.0);
#pragma omp for collapse(2) schedule(static)
        for (int k = 0; k < n; ++k)
            for (int iv = 0; iv < nv; ++iv)
                for (int iu = 0; iu < nu; ++iu) {
                    const double p = proj[(static_cast<size_t>(k) * nv + iv) * nu + iu];
                    siddon_ray(views[k], iu, iv, V, [&](long i, double l) { part[i] += p * l; });
                }
#pragma omp critical
        for (size_t i = 0; i < nvox; ++i) volume[i] += part[i];
    }
    return 0;
}

// BP_FDK_PseudoMatched: fdk_bp_kernel_matched_weight,
// src/FlatFpBp/BP/kernels/YkBpFdkKernel.cu:356-450, launched by
// fdk_pseudo_matched_bp_launch (:532-548) through BackOperator::apply
// (src/common/YkProjectionOperators.hpp:324-333).  Each voxel P takes the
// bilinear sample (zero outside the detector) at its projection (u, v) times
//     vox_x vox_y vox_z / (du dv) / |SDD_plane| * L^3 / |P - S|^2,
// L = |detS + u detU + v detV - S| the distance from the source to the
// detector point (YkFDKBpPrecompute.cu:104-122), du/dv of the first view.
// Voxels whose plane depth is not positive are skipped, as the reference
// skips den < 1e-8.
int orc_pseudo_bp(const orc_view* views, int n, int nu, int nv, const orc_volume* vol,
    const float* proj, double* volume, int flags)
{
    if (!valid_volume(vol) || !proj || !volume) return -1;
    std::vector<Derived> g;
    if (!derive(views, n, nu, nv, 6.28318530717958647692f, g)) return -2;
    const bool tex = (flags & 1) != 0;
    const orc_volume V = *vol;
    const double cell = static_cast<double>(V.vox_x) * V.vox_y * V.vox_z / (g[0].du * g[0].dv);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < V.nz; ++z)
        for (int y = 0; y < V.ny; ++y)
            for (int x = 0; x < V.nx; ++x) {
                const d3 P = md(vox_centre(x, V.nx, V.vox_x, V.center_x),
                    vox_centre(y, V.ny, V.vox_y, V.center_y),
                    vox_centre(z, V.nz, V.vox_z, V.center_z));
                double acc = 0.0;
                for (int i = 0; i < n; ++i) {
                    const Derived& d = g[i];
                    const d3 dir = subd(P, d.src);
                    const double dn = dotd(dir, d.n);
                    if (!(dn > 0.0)) continue;
                    double u, v, depth;
                    project_point(d, P, u, v, depth);
                    const d3 hit = addd(d.detS, addd(scaled(d.detU, u), scaled(d.detV, v)));
                    const d3 L = subd(hit, d.src);
                    const double L2 = dotd(L, L), lsq = dotd(dir, dir);
                    const double w = cell / std::fabs(d.plane) * L2 * std::sqrt(L2) / lsq;
                    acc += w * bilerp_zero(proj + static_cast<size_t>(i) * nu * nv, nu, nv, u, v, tex);
                }
                volume[(static_cast<size_t>(z) * V.ny + y) * V.nx + x] = acc;
            }
    return 0;
}

int orc_fdk(const orc_view* views, int n, int nu, int nv, float range,
    const orc_volume* vol, const orc_filter* filter, const float* proj,
    double* volume_out, int flags)
{
    return orc_fdk_weighted(views, n, nu, nv, range, vol, filter, proj, nullptr, volume_out, flags);
}

int orc_fdk_weighted(const orc_view* views, int n, int nu, int nv, float range,
    const orc_volume* vol, const orc_filter* filter, const float* proj,
    const double* row_weights, double* volume_out, int flags)
{
    if (!valid_volume(vol)) return -1;
    std::vector<double> flt(static_cast<size_t>(n) * nu * nv);
    int rc = orc_fdk_filter_weighted(views, n, nu, nv, range, filter, proj, row_weights, flt.data());
    if (rc) return rc;
    std::fill(volume_out, volume_out + static_cast<size_t>(vol->nx) * vol->ny * vol->nz, 0.0);
    return orc_fdk_backproject(views, n, nu, nv, range, vol, flt.data(), volume_out, flags);
}

// FP32 transcription: the same loops with float storage and float
// arithmetic for the per-voxel work (coefficients derived in FP64 as above).
int orc_fdk_fp32(const orc_view* views, int n, int nu, int nv, float range,
    const orc_volume* vol, const orc_filter* filter, const float* proj,
    float* volume_out)
{
    if (!valid_volume(vol) || !filter || !proj || !volume_out) return -1;
    std::vector<Derived> g;
    if (!derive(views, n, nu, nv, range, g)) return -2;
    std::vector<double> hd;
    ramp_kernel(nu, g[0].du, *filter, hd);
    std::vector<float> h(hd.begin(), hd.end());
    const int N = padded_n(nu);
    std::vector<float> flt(static_cast<size_t>(n) * nu * nv);
#pragma omp parallel
    {
        std::vector<float> row(nu);
#pragma omp for schedule(static)
        for (long r = 0; r < static_cast<long>(n) * nv; ++r) {
            const int i = static_cast<int>(r / nv);
            const int iv = static_cast<int>(r % nv);
            const Derived& d = g[i];
            const float wgeom = static_cast<float>(d.dsd / d.sid / 2.0);
            const float dsd = static_cast<float>(d.dsd);
            const float* src = proj + static_cast<size_t>(r) * nu;
            for (int iu = 0; iu < nu; ++iu) {
                const float qx = static_cast<float>(d.detS.x + iu * d.detU.x + iv * d.detV.x - d.src.x);
                const float qy = static_cast<float>(d.detS.y + iu * d.detU.y + iv * d.detV.y - d.src.y);
                const float qz = static_cast<float>(d.detS.z + iu * d.detU.z + iv * d.detV.z - d.src.z);
                const bool placed = (iu + d.startU) >= 0 && (iu + d.startU) < N;
                row[iu] = placed ? src[iu] * (dsd / std::sqrt(qx * qx + qy * qy + qz * qz)) * wgeom : 0.f;
            }
            float* dst = flt.data() + static_cast<size_t>(r) * nu;
            for (int j = 0; j < nu; ++j) {
                const bool valid = (j + d.startU) >= 0 && (j + d.startU) < N;
                float s = 0.f;
                if (valid)
                    for (int k = 0; k < nu; ++k) s += row[k] * h[j - k + nu - 1];
                dst[j] = s;
            }
        }
    }
    struct C { float cu[4], cv[4], cd[4], cr[4]; float w; };
    std::vector<C> co(n);
    for (int i = 0; i < n; ++i) {
        const Derived& d = g[i];
        // affine rows of the 3x4 projection (YkFDKBpPrecompute.cu:40-87)
        const double sn = dotd(d.src, d.n), su = dotd(d.src, d.detU), sv = dotd(d.src, d.detV);
        const double ou = dotd(subd(d.detS, d.src), d.detU), ov = dotd(subd(d.detS, d.src), d.detV);
        const double P = d.plane;
        const double cux[4] = {P * d.detU.x - ou * d.n.x, P * d.detU.y - ou * d.n.y,
            P * d.detU.z - ou * d.n.z, -P * su + ou * sn};
        const double cvx[4] = {P * d.detV.x - ov * d.n.x, P * d.detV.y - ov * d.n.y,
            P * d.detV.z - ov * d.n.z, -P * sv + ov * sn};
        for (int k = 0; k < 4; ++k) {
            co[i].cu[k] = static_cast<float>((cux[k] * d.VV - cvx[k] * d.UV) * d.inv_gram);
            co[i].cv[k] = static_cast<float>((-cux[k] * d.UV + cvx[k] * d.UU) * d.inv_gram);
        }
        const double cd[4] = {d.n.x, d.n.y, d.n.z, -sn};
        const double cr[4] = {d.radial.x, d.radial.y, d.radial.z, -dotd(d.src, d.radial)};
        for (int k = 0; k < 4; ++k) { co[i].cd[k] = static_cast<float>(cd[k]); co[i].cr[k] = static_cast<float>(cr[k]); }
        co[i].w = static_cast<float>(d.sid * d.sid * d.dtheta * d.fscale);
    }
    const orc_volume V = *vol;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < V.nz; ++z)
        for (int y = 0; y < V.ny; ++y)
            for (int x = 0; x < V.nx; ++x) {
                const float X = static_cast<float>(vox_centre(x, V.nx, V.vox_x, V.center_x));
                const float Y = static_cast<float>(vox_centre(y, V.ny, V.vox_y, V.center_y));
                const float Z = static_cast<float>(vox_centre(z, V.nz, V.vox_z, V.center_z));
                float acc = 0.f;
                for (int i = 0; i < n; ++i) {
                    const C& c = co[i];
                    const float den = c.cd[3] + X * c.cd[0] + Y * c.cd[1] + Z * c.cd[2];
                    const float un = c.cu[3] + X * c.cu[0] + Y * c.cu[1] + Z * c.cu[2];
                    const float vn = c.cv[3] + X * c.cv[0] + Y * c.cv[1] + Z * c.cv[2];
                    const float dp = c.cr[3] + X * c.cr[0] + Y * c.cr[1] + Z * c.cr[2];
                    const float u = un / den, v = vn / den;
                    const float fu = std::floor(u), fv = std::floor(v);
                    const int iu = static_cast<int>(fu), iv = static_cast<int>(fv);
                    const float au = u - fu, av = v - fv;
                    const float* img = flt.data() + static_cast<size_t>(i) * nu * nv;
                    auto at = [&](int xx, int yy) -> float {
                        if (xx < 0 || yy < 0 || xx >= nu || yy >= nv) return 0.f;
                        return img[static_cast<size_t>(yy) * nu + xx];
                    };
                    const float val = (1 - av) * ((1 - au) * at(iu, iv) + au * at(iu + 1, iv)) +
                        av * ((1 - au) * at(iu, iv + 1) + au * at(iu + 1, iv + 1));
                    acc += val * (c.w / (dp * dp));
                }
                volume_out[(static_cast<size_t>(z) * V.ny + y) * V.nx + x] = acc;
            }
    return 0;
}

int orc_joseph_main_axes(const orc_view* views, int n, int nu, int nv, int* axes)
{
    for (int i = 0; i < n; ++i) {
        axes[i] = main_axis_float(views[i], nu, nv);
        if (axes[i] < 0) return -1;
    }
    return 0;
}

// Joseph forward projection (src/FlatFpBp/FP/kernels/YkFPKernels.cu:10-202,
// launch and 256-slice segmentation :325-362,530-565): one sample per voxel
// centre of the main axis, bilinear with zero border on the minor axes.
int orc_joseph_fp(const orc_view* views, int n, int nu, int nv,
    const orc_volume* vol, const float* volume, double* proj, int flags)
{
    if (!valid_volume(vol) || !volume || !proj) return -1;
    std::vector<JosephView> jv;
    if (!joseph_views(views, n, nu, nv, *vol, jv)) return -2;
    const bool tex = (flags & 1) != 0;
    const orc_volume V = *vol;
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int i = 0; i < n; ++i)
        for (int iv = 0; iv < nv; ++iv) {
            const JosephView& j = jv[i];
            for (int iu = 0; iu < nu; ++iu) {
                const Ray r = ray_params(j, iu, iv);
                double acc = 0.0;
                if (r.ok) {
                    for (int s = 0; s < j.n0; ++s) {
                        const double c0 = s - 0.5 * (j.n0 - 1);
                        const double f1 = r.a1 * c0 + r.b1 + 0.5 * (j.n1 - 1);
                        const double f2 = r.a2 * c0 + r.b2 + 0.5 * (j.n2 - 1);
                        const double fl1 = std::floor(f1), fl2 = std::floor(f2);
                        const int i1 = static_cast<int>(fl1), i2 = static_cast<int>(fl2);
                        double w1 = f1 - fl1, w2 = f2 - fl2;
                        if (tex) { w1 = tex_frac(w1); w2 = tex_frac(w2); }
                        auto at = [&](int a, int b) -> double {
                            if (a < 0 || b < 0 || a >= j.n1 || b >= j.n2) return 0.0;
                            return volume[vox_index(V, j.axis, s, a, b)];
                        };
                        acc += (1 - w2) * ((1 - w1) * at(i1, i2) + w1 * at(i1 + 1, i2)) +
                            w2 * ((1 - w1) * at(i1, i2 + 1) + w1 * at(i1 + 1, i2 + 1));
                    }
                    acc *= r.len;
                }
                proj[(static_cast<size_t>(i) * nv + iv) * nu + iu] = acc;
            }
        }
    return 0;
}

namespace {
// Scatter transpose of orc_joseph_fp (the form of
// src/FlatFpBp/BP/kernels/YkBPJosephKernel.cu:12-113).  ref_weight selects
// the reference's vox0*sqrt(1+a1^2+a2^2) factor (:75-76).
int joseph_bp_impl(const orc_view* views, int n, int nu, int nv,
    const orc_volume* vol, const float* proj, double* volume, bool ref_weight)
{
    if (!valid_volume(vol) || !proj || !volume) return -1;
    std::vector<JosephView> jv;
    if (!joseph_views(views, n, nu, nv, *vol, jv)) return -2;
    const orc_volume V = *vol;
    std::fill(volume, volume + static_cast<size_t>(V.nx) * V.ny * V.nz, 0.0);
    std::vector<Ray> rays(static_cast<size_t>(nu) * nv);
    for (int i = 0; i < n; ++i) {
        const JosephView& j = jv[i];
        for (int iv = 0; iv < nv; ++iv)
            for (int iu = 0; iu < nu; ++iu) {
                Ray r = ray_params(j, iu, iv);
                if (ref_weight && r.ok)
                    r.len = j.v0 * std::sqrt(1.0 + r.a1 * r.a1 + r.a2 * r.a2);
                rays[static_cast<size_t>(iv) * nu + iu] = r;
            }
        const float* p = proj + static_cast<size_t>(i) * nu * nv;
        // each main-axis slice owns disjoint voxels: parallel over slices
#pragma omp parallel for schedule(static)
        for (int s = 0; s < j.n0; ++s) {
            const double c0 = s - 0.5 * (j.n0 - 1);
            for (int iv = 0; iv < nv; ++iv)
                for (int iu = 0; iu < nu; ++iu) {
                    const Ray& r = rays[static_cast<size_t>(iv) * nu + iu];
                    if (!r.ok) continue;
                    const double q = static_cast<double>(p[static_cast<size_t>(iv) * nu + iu]) * r.len;
                    if (q == 0.0) continue;
                    const double f1 = r.a1 * c0 + r.b1 + 0.5 * (j.n1 - 1);
                    const double f2 = r.a2 * c0 + r.b2 + 0.5 * (j.n2 - 1);
                    const double fl1 = std::floor(f1), fl2 = std::floor(f2);
                    const int i1 = static_cast<int>(fl1), i2 = static_cast<int>(fl2);
                    if (i1 < -1 || i1 >= j.n1 || i2 < -1 || i2 >= j.n2) continue;
                    const double w1 = f1 - fl1, w2 = f2 - fl2;
                    auto add = [&](int a, int b, double w) {
                        if (a < 0 || b < 0 || a >= j.n1 || b >= j.n2) return;
                        volume[vox_index(V, j.axis, s, a, b)] += q * w;
                    };
                    add(i1, i2, (1 - w1) * (1 - w2));
                    add(i1 + 1, i2, w1 * (1 - w2));
                    add(i1, i2 + 1, (1 - w1) * w2);
                    add(i1 + 1, i2 + 1, w1 * w2);
                }
        }
    }
    return 0;
}
} // namespace

int orc_joseph_bp(const orc_view* views, int n, int nu, int nv,
    const orc_volume* vol, const float* proj, double* volume)
{
    return joseph_bp_impl(views, n, nu, nv, vol, proj, volume, false);
}

int orc_joseph_bp_refweight(const orc_view* views, int n, int nu, int nv,
    const orc_volume* vol, const float* proj, double* volume)
{
    return joseph_bp_impl(views, n, nu, nv, vol, proj, volume, true);
}

// Seeded ellipsoid parameters: centres U[-r,r], semi-axes U[a0,a1], three
// rotation angles U[0,2pi), additive value U[v0,v1].
int orc_random_ellipsoids(uint64_t seed, int count, double cr, double a0,
    double a1, double v0, double v1, orc_ellipsoid* out)
{
    std::mt19937_64 g(splitmix(seed));
    for (int i = 0; i < count; ++i) {
        orc_ellipsoid& e = out[i];
        e.cx = -cr + 2 * cr * uni01(g);
        e.cy = -cr + 2 * cr * uni01(g);
        e.cz = -cr + 2 * cr * uni01(g);
        e.ax = a0 + (a1 - a0) * uni01(g);
        e.ay = a0 + (a1 - a0) * uni01(g);
        e.az = a0 + (a1 - a0) * uni01(g);
        e.phi = 2 * kPi * uni01(g);
        e.theta = 2 * kPi * uni01(g);
        e.psi = 2 * kPi * uni01(g);
        e.value = v0 + (v1 - v0) * uni01(g);
    }
    return 0;
}

int orc_random_spheres(uint64_t seed, int count, double cr, double r0, double r1,
    double value, orc_ellipsoid* out)
{
    std::mt19937_64 g(splitmix(seed ^ 0x5EEDull));
    for (int i = 0; i < count; ++i) {
        orc_ellipsoid& e = out[i];
        e.cx = -cr + 2 * cr * uni01(g);
        e.cy = -cr + 2 * cr * uni01(g);
        e.cz = -cr + 2 * cr * uni01(g);
        const double r = r0 + (r1 - r0) * uni01(g);
        e.ax = e.ay = e.az = r;
        e.phi = e.theta = e.psi = 0.0;
        e.value = value;
    }
    return 0;
}

// Centre-sampled voxelisation (as Yktest/YkTestPhantoms.hpp:81-99 samples
// its ellipsoids); rotation R = Rz(phi) Ry(theta) Rz(psi).
int orc_voxelize(const orc_volume* vol, const orc_ellipsoid* e, int count, float* out)
{
    if (!valid_volume(vol) || (count > 0 && !e) || !out) return -1;
    struct R { double m[9]; };
    std::vector<R> rot(count);
    for (int k = 0; k < count; ++k) {
        const double c1 = std::cos(e[k].phi), s1 = std::sin(e[k].phi);
        const double c2 = std::cos(e[k].theta), s2 = std::sin(e[k].theta);
        const double c3 = std::cos(e[k].psi), s3 = std::sin(e[k].psi);
        // Rz(phi)*Ry(theta)*Rz(psi)
        const double m[9] = {
            c1 * c2 * c3 - s1 * s3, -c1 * c2 * s3 - s1 * c3, c1 * s2,
            s1 * c2 * c3 + c1 * s3, -s1 * c2 * s3 + c1 * c3, s1 * s2,
            -s2 * c3, s2 * s3, c2};
        std::copy(m, m + 9, rot[k].m);
    }
    const orc_volume V = *vol;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < V.nz; ++z)
        for (int y = 0; y < V.ny; ++y)
            for (int x = 0; x < V.nx; ++x) {
                const double px = vox_centre(x, V.nx, V.vox_x, V.center_x);
                const double py = vox_centre(y, V.ny, V.vox_y, V.center_y);
                const double pz = vox_centre(z, V.nz, V.vox_z, V.center_z);
                double val = 0.0;
                for (int k = 0; k < count; ++k) {
                    const double dx = px - e[k].cx, dy = py - e[k].cy, dz = pz - e[k].cz;
                    const double* m = rot[k].m;
                    // local = R^T d
                    const double lx = m[0] * dx + m[3] * dy + m[6] * dz;
                    const double ly = m[1] * dx + m[4] * dy + m[7] * dz;
                    const double lz = m[2] * dx + m[5] * dy + m[8] * dz;
                    const double q = lx * lx / (e[k].ax * e[k].ax) + ly * ly / (e[k].ay * e[k].ay) +
                        lz * lz / (e[k].az * e[k].az);
                    if (q <= 1.0) val += e[k].value;
                }
                out[(static_cast<size_t>(z) * V.ny + y) * V.nx + x] = static_cast<float>(val);
            }
    return 0;
}

// p' = -ln(max(Poisson(I0 exp(-p)), 1) / I0)
int orc_poisson_noise(float* proj, size_t n, double i0, uint64_t seed)
{
    if (!proj || !(i0 > 0)) return -1;
    const size_t block = 65536;
    const long nb = static_cast<long>((n + block - 1) / block);
#pragma omp parallel for schedule(dynamic, 4)
    for (long b = 0; b < nb; ++b) {
        std::mt19937_64 g(splitmix(seed * 0x100000001B3ull + static_cast<uint64_t>(b)));
        const size_t e = std::min(n, static_cast<size_t>(b + 1) * block);
        for (size_t k = static_cast<size_t>(b) * block; k < e; ++k) {
            const long c = poisson(g, i0 * std::exp(-static_cast<double>(proj[k])));
            proj[k] = static_cast<float>(-std::log(std::max<double>(c, 1.0) / i0));
        }
    }
    return 0;
}

int orc_uniform(float* out, size_t n, double lo, double hi, uint64_t seed)
{
    const size_t block = 65536;
    const long nb = static_cast<long>((n + block - 1) / block);
#pragma omp parallel for schedule(static)
    for (long b = 0; b < nb; ++b) {
        std::mt19937_64 g(splitmix(seed * 0x9E3779B1ull + static_cast<uint64_t>(b)));
        const size_t e = std::min(n, static_cast<size_t>(b + 1) * block);
        for (size_t k = static_cast<size_t>(b) * block; k < e; ++k)
            out[k] = static_cast<float>(lo + (hi - lo) * uni01(g));
    }
    return 0;
}

// Box-Muller over mt19937_64
int orc_normal(float* out, size_t n, uint64_t seed)
{
    const size_t block = 65536;
    const long nb = static_cast<long>((n + block - 1) / block);
#pragma omp parallel for schedule(static)
    for (long b = 0; b < nb; ++b) {
        std::mt19937_64 g(splitmix(seed * 0xC2B2AE3Dull + static_cast<uint64_t>(b)));
        const size_t e = std::min(n, static_cast<size_t>(b + 1) * block);
        for (size_t k = static_cast<size_t>(b) * block; k < e; k += 2) {
            double u1 = uni01(g);
            if (u1 < 1e-300) u1 = 1e-300;
            const double u2 = uni01(g);
            const double r = std::sqrt(-2.0 * std::log(u1));
            out[k] = static_cast<float>(r * std::cos(2 * kPi * u2));
            if (k + 1 < e) out[k + 1] = static_cast<float>(r * std::sin(2 * kPi * u2));
        }
    }
    return 0;
}

int orc_mt19937_uniform_pm1(float* out, size_t n, uint32_t seed)
{
    std::mt19937 g(seed);
    std::uniform_real_distribution<float> d(-1.f, 1.f);
    for (size_t i = 0; i < n; ++i) out[i] = d(g);
    return 0;
}

} // extern "C"
