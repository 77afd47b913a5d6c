// Host-side geometry for libykb: the regular circular builder (float, as the
// reference builders), FDK derived quantities and projection coefficients
// (FP64), the analytic ramp kernel and the Joseph per-view data.
#include "ykb_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace ykb {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr float kTwoPiF = 6.28318530717958647692f;

struct fv3 { float x, y, z; };
inline fv3 f3(float x, float y, float z) { return {x, y, z}; }
inline float fdot(fv3 a, fv3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline fv3 fcross(fv3 a, fv3 b)
{ return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline fv3 fadd(fv3 a, fv3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline fv3 fsub(fv3 a, fv3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline fv3 fscale(fv3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
inline fv3 fnormalized(fv3 a)
{
    const float l2 = fdot(a, a);
    if (!(l2 > 0.f)) return f3(0.f, 0.f, 0.f);
    return fscale(a, 1.f / std::sqrt(l2));
}
// rotation of v about axis by angle (Rodrigues), as
// include/YKCBCT/geometry/YkDetectorGeometryBuilders.hpp:37-44
inline fv3 frotate(fv3 v, fv3 axis, float angle)
{
    const fv3 k = fnormalized(axis);
    const float c = std::cos(angle), s = std::sin(angle);
    return fadd(fadd(fscale(v, c), fscale(fcross(k, v), s)), fscale(k, fdot(k, v) * (1.f - c)));
}
inline fv3 frotz(fv3 v, float angle)
{
    const float c = std::cos(angle), s = std::sin(angle);
    return f3(c * v.x - s * v.y, s * v.x + c * v.y, v.z);
}

inline dvec3 d3(double x, double y, double z) { return {x, y, z}; }
inline dvec3 dof(const ykb_float4& v) { return d3(v.x, v.y, v.z); }
inline double ddot(dvec3 a, dvec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline dvec3 dcross(dvec3 a, dvec3 b)
{ return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline dvec3 dadd(dvec3 a, dvec3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline dvec3 dsub(dvec3 a, dvec3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline dvec3 dscale(dvec3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
inline double dlen(dvec3 a) { return std::sqrt(ddot(a, a)); }

inline bool finite4(const ykb_float4& v)
{ return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

} // namespace

int padded_fft_length(int nu)
{
    int n = 1;
    while (n < 2 * nu) n <<= 1;
    return n;
}

VolumeGrid make_grid(const ykb_volume& v)
{
    VolumeGrid g{};
    g.nx = v.nx; g.ny = v.ny; g.nz = v.nz;
    g.vx = v.vox_x; g.vy = v.vox_y; g.vz = v.vox_z;
    g.ox = static_cast<double>(v.center_x) - 0.5 * (v.nx - 1) * g.vx;
    g.oy = static_cast<double>(v.center_y) - 0.5 * (v.ny - 1) * g.vy;
    g.oz = static_cast<double>(v.center_z) - 0.5 * (v.nz - 1) * g.vz;
    return g;
}

// Regular circular trajectory with a flat detector; the float operation
// sequence of buildCircularTrajectory/buildRegularAngles
// (include/YKCBCT/geometry/YkSystemGeometry.hpp:37-73),
// buildScannerViewFramesImpl (YkTrajectoryGeometryBuilder.hpp:29-67) and
// detectorAxes/buildFlatProjectionGeometry (YkDetectorGeometryBuilders.hpp:46-107),
// so the per-view geometry is bit-identical to the reference builders.
bool build_circular_flat(const ykb_circular_flat& s, ykb_cone_view* out,
    std::string& why)
{
    if (!(s.total_views > 0 && s.views_per_turn >= 2 &&
          (s.rotation_direction == 1 || s.rotation_direction == -1) &&
          s.sid_mm > 0.f && s.sdd_mm > s.sid_mm && std::isfinite(s.start_angle_rad) &&
          std::isfinite(s.z_mm) && std::isfinite(s.source_offset_mm[0]) &&
          std::isfinite(s.source_offset_mm[1]) && std::isfinite(s.source_offset_mm[2]))) {
        why = "invalid regular circular scan (views, direction, SID/SDD or offsets)";
        return false;
    }
    if (s.channels <= 0 || s.rows <= 0 || !(s.channel_size_mm > 0.f) ||
        !(s.row_size_mm > 0.f) || !std::isfinite(s.offset_unv_mm[0]) ||
        !std::isfinite(s.offset_unv_mm[1]) || !std::isfinite(s.offset_unv_mm[2]) ||
        !std::isfinite(s.tilt_u_rad) || !std::isfinite(s.tilt_v_rad) ||
        !std::isfinite(s.tilt_n_rad)) {
        why = "invalid flat detector (size, pitch or pose)";
        return false;
    }
    const float step = static_cast<float>(s.rotation_direction) * kTwoPiF /
        static_cast<float>(s.views_per_turn);
    const float detector_distance = s.sdd_mm - s.sid_mm;
    const float cu = 0.5f * (s.channels - 1);
    const float cv = 0.5f * (s.rows - 1);
    for (int i = 0; i < s.total_views; ++i) {
        const float angle = s.start_angle_rad + i * step;
        const fv3 zshift = f3(0.f, 0.f, s.z_mm);
        const fv3 src_local = f3(s.source_offset_mm[0], -s.sid_mm + s.source_offset_mm[1],
            s.source_offset_mm[2]);
        const fv3 det_local = f3(0.f, detector_distance, 0.f);
        const fv3 rs = frotz(src_local, angle), rd = frotz(det_local, angle);
        const fv3 source = f3(rs.x + zshift.x, rs.y + zshift.y, rs.z + zshift.z);
        const fv3 principal = f3(rd.x + zshift.x, rd.y + zshift.y, rd.z + zshift.z);
        fv3 u = frotz(f3(1.f, 0.f, 0.f), angle);
        fv3 v = f3(0.f, 0.f, 1.f);
        fv3 n = frotz(f3(0.f, -1.f, 0.f), angle);
        v = frotate(v, u, s.tilt_u_rad);
        n = frotate(n, u, s.tilt_u_rad);
        u = frotate(u, v, s.tilt_v_rad);
        n = frotate(n, v, s.tilt_v_rad);
        u = frotate(u, n, s.tilt_n_rad);
        v = frotate(v, n, s.tilt_n_rad);
        u = fnormalized(u);
        v = fnormalized(v);
        n = fnormalized(fcross(u, v));
        if (fdot(n, fsub(source, principal)) < 0.f) n = fscale(n, -1.f);
        const fv3 centre = fadd(principal, fadd(fscale(u, s.offset_unv_mm[0]),
            fadd(fscale(n, s.offset_unv_mm[1]), fscale(v, s.offset_unv_mm[2]))));
        const fv3 du = fscale(u, s.channel_size_mm);
        const fv3 dv = fscale(v, s.row_size_mm);
        const fv3 start = fsub(fsub(centre, fscale(du, cu)), fscale(dv, cv));
        out[i].src = {source.x, source.y, source.z, 0.f};
        out[i].detS = {start.x, start.y, start.z, 0.f};
        out[i].detU = {du.x, du.y, du.z, 0.f};
        out[i].detV = {dv.x, dv.y, dv.z, 0.f};
        out[i].angle = {angle, 0.f, 0.f, 0.f};
    }
    return true;
}

// FDK derived geometry in FP64.  Definitions follow
// src/Reconstruction/Analytic/Circular/Flat/FDK/YkFDKVecGeoDerived.hpp:
//  - theta unwrap and central-difference dtheta (:158-184),
//  - fScaleDTheta = 2pi / scan range (:94),
//  - SID via the radial ray from the source to the rotation axis (:194-209),
//  - detector normal/plane distance from deriveProjectionFrame
//    (include/YKCBCT/geometry/YkProjectionGeometry.hpp:114-194),
//  - principal point, DSD and pixel offsets (:257-304);
// and validateApproximateFdkGeometry_ rejections
// (src/Reconstruction/Analytic/Circular/Flat/FDK/YkFdkPipeline.hpp:665-866).
bool derive_fdk_geometry(const ykb_cone_view* views, int n, int nu, int nv,
    float scan_range, std::vector<FdkDerived>& out, std::string& why)
{
    if (n <= 0 || nu <= 0 || nv <= 0) { why = "empty view sequence or detector"; return false; }
    if (!(scan_range > 0.f) || !std::isfinite(scan_range)) { why = "scan range must be positive"; return false; }
    out.assign(n, FdkDerived{});
    std::vector<double> th(n);
    for (int i = 0; i < n; ++i) {
        if (!finite4(views[i].src) || !finite4(views[i].detS) || !finite4(views[i].detU) ||
            !finite4(views[i].detV) || !std::isfinite(views[i].angle.x)) {
            why = "non-finite view geometry";
            return false;
        }
        th[i] = views[i].angle.x;
    }
    for (int i = 1; i < n; ++i) {
        if (std::fabs(static_cast<double>(views[i].angle.x) - views[i - 1].angle.x) < 1e-5) {
            why = "repeated adjacent view angles: dtheta is undefined";
            return false;
        }
        double t = th[i];
        while (t - th[i - 1] > kPi) t -= 2 * kPi;
        while (t - th[i - 1] < -kPi) t += 2 * kPi;
        th[i] = t;
    }
    const int padded = padded_fft_length(nu);
    for (int i = 0; i < n; ++i) {
        FdkDerived& g = out[i];
        g.theta = th[i];
        double dt = n <= 1 ? 1e-8 : i == 0 ? th[1] - th[0] : i == n - 1 ? th[n - 1] - th[n - 2]
            : 0.5 * (th[i + 1] - th[i - 1]);
        dt = std::fabs(dt);
        g.dtheta = std::max(dt, 1e-8);
        g.fscale = 2.0 * kPi / static_cast<double>(scan_range);
        g.src = dof(views[i].src); g.detS = dof(views[i].detS);
        g.detU = dof(views[i].detU); g.detV = dof(views[i].detV);
        g.du = dlen(g.detU); g.dv = dlen(g.detV);
        if (!(g.du > 0) || !(g.dv > 0)) { why = "degenerate detector pixel axes"; return false; }
        const dvec3 centre = dadd(g.detS, dadd(dscale(g.detU, 0.5 * (nu - 1)), dscale(g.detV, 0.5 * (nv - 1))));
        const dvec3 cdir = dsub(centre, g.src);
        dvec3 nrm = dcross(g.detV, g.detU);
        const double nl = dlen(nrm);
        if (!(nl > 1e-12) || !(dlen(cdir) > 1e-9)) { why = "degenerate detector frame"; return false; }
        nrm = dscale(nrm, 1.0 / nl);
        if (ddot(nrm, cdir) < 0) nrm = dscale(nrm, -1.0);
        g.normal = nrm;
        g.plane = ddot(dsub(g.detS, g.src), nrm);
        if (!(g.plane > 1e-9)) { why = "source lies on or behind the detector plane"; return false; }
        const dvec3 ray = d3(-g.src.x, -g.src.y, 0.0);  // closest axis point (0,0,src.z)
        const double rl = dlen(ray);
        if (!(rl > 1e-9)) { why = "source on the rotation axis"; return false; }
        g.sid = rl;
        g.radial = dscale(ray, 1.0 / rl);
        const double den = ddot(g.radial, nrm);
        if (std::fabs(den) < 1e-12) { why = "radial ray parallel to the detector"; return false; }
        const double t = g.plane / den;
        if (!(t > 0)) { why = "detector behind the source along the radial ray"; return false; }
        const dvec3 pp = dadd(g.src, dscale(g.radial, t));
        g.dsd = dlen(dsub(pp, g.src));
        g.UU = ddot(g.detU, g.detU); g.VV = ddot(g.detV, g.detV); g.UV = ddot(g.detU, g.detV);
        const double gram = g.UU * g.VV - g.UV * g.UV;
        if (std::fabs(gram) < 1e-20) { why = "singular detector basis"; return false; }
        g.inv_gram = 1.0 / gram;
        const dvec3 D = dsub(pp, g.detS);
        const double DU = ddot(D, g.detU), DV = ddot(D, g.detV);
        g.off_u = (DU * g.VV - DV * g.UV) * g.inv_gram - 0.5 * (nu - 1);
        g.off_v = (-DU * g.UV + DV * g.UU) * g.inv_gram - 0.5 * (nv - 1);
        // startU: the integer placement of the row inside the padded FFT row,
        // decided in float exactly as fp_computeStartU
        // (.../FDK/kernels/YkFDKFilterHelpers.cuh:37-42)
        const float axis = (nu - 1) * 0.5f + static_cast<float>(g.off_u);
        g.start_u = static_cast<int>(lrintf(padded * 0.5f - axis));
    }
    return true;
}

// Affine projection rows in FP64 (the algebra of fdk_precompute_coeffs_kernel,
// .../FDK/kernels/YkFDKBpPrecompute.cu:14-138, kept in double) and the
// per-view preweight/placement records.
// Parker short-scan weights per (view, column), FP64, with the range/pi
// scale folded in.  Restates .../FDK/kernels/YkFDKParkerKernels.cu:46-110
// (fan angle of column u on the centre row against the radial ray, Gamma =
// the larger edge |fan| of the view, sin^2 ramps of width 2(Gamma +- gamma)),
// the relative angle of pk_uploadAngles (:117-138) and the coverage check of
// FdkPipeline::validateParkerCoverage_ (YkFdkPipeline.hpp:597-635).
bool build_parker_weights(const std::vector<FdkDerived>& g, const ykb_cone_view* views, int nu,
    int nv, double scan_range, double start_angle, int direction, std::vector<float>& w,
    std::string& why)
{
    const double pi = 3.14159265358979323846;
    if (direction != 1 && direction != -1) { why = "rotation direction must be +1 or -1"; return false; }
    if (scan_range >= 2.0 * pi - 1e-5) {
        why = "Parker weighting needs a short scan (range below 2 pi)";
        return false;
    }
    const int n = static_cast<int>(g.size());
    const double cv = 0.5 * (nv - 1);
    double max_fan = 0.0;
    for (const FdkDerived& d : g) {
        const double cu = 0.5 * (nu - 1);
        const double px = d.detS.x + cu * d.detU.x + cv * d.detV.x - d.src.x;
        const double py = d.detS.y + cu * d.detU.y + cv * d.detV.y - d.src.y;
        for (double u : {0.0, static_cast<double>(nu - 1)}) {
            const double rx = d.detS.x + u * d.detU.x + cv * d.detV.x - d.src.x;
            const double ry = d.detS.y + u * d.detU.y + cv * d.detV.y - d.src.y;
            max_fan = std::max(max_fan, std::fabs(std::atan2(rx * py - ry * px, rx * px + ry * py)));
        }
    }
    if (scan_range + 1e-5 < pi + 2.0 * max_fan) {
        why = "short scan too short for Parker weighting (needs pi + 2 x fan angle)";
        return false;
    }
    const double scale = scan_range / pi, eps = 1e-6;
    w.assign(static_cast<size_t>(n) * nu, 0.f);
    for (int i = 0; i < n; ++i) {
        const FdkDerived& d = g[i];
        auto fan = [&](double u) {
            const double rx = d.detS.x + u * d.detU.x + cv * d.detV.x - d.src.x;
            const double ry = d.detS.y + u * d.detU.y + cv * d.detV.y - d.src.y;
            return std::atan2(rx * d.radial.y - ry * d.radial.x, rx * d.radial.x + ry * d.radial.y);
        };
        const double Gamma = std::max(std::fabs(fan(0.0)), std::fabs(fan(nu - 1.0)));
        double beta = direction * (static_cast<double>(views[i].angle.x) - start_angle);
        while (beta < 0.0) beta += 2.0 * pi;
        while (beta >= 2.0 * pi) beta -= 2.0 * pi;
        for (int u = 0; u < nu; ++u) {
            const double gamma = direction * fan(u);
            const double t1 = 2.0 * (Gamma + gamma), t2 = pi + 2.0 * gamma, t3 = pi + 2.0 * Gamma;
            double x = 0.0;
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
            }
            w[static_cast<size_t>(i) * nu + u] = static_cast<float>(x * scale);
        }
    }
    return true;
}

void build_fdk_coefficients(const std::vector<FdkDerived>& g, int nu,
    std::vector<FdkViewCoef>& coef, std::vector<FdkPreweightView>& pw, bool& axial)
{
    const int n = static_cast<int>(g.size());
    const int padded = padded_fft_length(nu);
    coef.assign(n, FdkViewCoef{});
    pw.assign(n, FdkPreweightView{});
    axial = true;
    for (int i = 0; i < n; ++i) {
        const FdkDerived& d = g[i];
        const double sn = ddot(d.src, d.normal), su = ddot(d.src, d.detU), sv = ddot(d.src, d.detV);
        const double ou = ddot(dsub(d.detS, d.src), d.detU), ov = ddot(dsub(d.detS, d.src), d.detV);
        const double P = d.plane;
        const double ru[4] = {P * d.detU.x - ou * d.normal.x, P * d.detU.y - ou * d.normal.y,
            P * d.detU.z - ou * d.normal.z, -P * su + ou * sn};
        const double rv[4] = {P * d.detV.x - ov * d.normal.x, P * d.detV.y - ov * d.normal.y,
            P * d.detV.z - ov * d.normal.z, -P * sv + ov * sn};
        FdkViewCoef& c = coef[i];
        for (int k = 0; k < 4; ++k) {
            c.cu[k] = (ru[k] * d.VV - rv[k] * d.UV) * d.inv_gram;
            c.cv[k] = (-ru[k] * d.UV + rv[k] * d.UU) * d.inv_gram;
        }
        c.cd[0] = d.normal.x; c.cd[1] = d.normal.y; c.cd[2] = d.normal.z; c.cd[3] = -sn;
        c.cr[0] = d.radial.x; c.cr[1] = d.radial.y; c.cr[2] = d.radial.z;
        c.cr[3] = -ddot(d.src, d.radial);
        c.wbase = d.sid * d.sid * d.dtheta * d.fscale;
        // u, denominator and depth independent of z: a thread walking a
        // z-column keeps its detector column and weight
        if (c.cu[2] != 0.0 || c.cd[2] != 0.0 || c.cr[2] != 0.0) axial = false;

        FdkPreweightView& p = pw[i];
        p.src[0] = d.src.x; p.src[1] = d.src.y; p.src[2] = d.src.z;
        p.detS[0] = d.detS.x; p.detS[1] = d.detS.y; p.detS[2] = d.detS.z;
        p.detU[0] = d.detU.x; p.detU[1] = d.detU.y; p.detU[2] = d.detU.z;
        p.detV[0] = d.detV.x; p.detV[1] = d.detV.y; p.detV[2] = d.detV.z;
        p.dsd = d.dsd;
        p.wgeom = d.dsd / d.sid / 2.0;
        // _fp_pad_kernel places input j at padded index j + startU, and
        // _fp_crop_kernel reads output j from j + startU
        // (.../FDK/kernels/YkFDKFilterKernels.cu:32-95): samples outside
        // [0, padded) are dropped (input) or read as zero (output).
        p.in_lo = std::max(0, -d.start_u);
        p.in_hi = std::min(nu, padded - d.start_u);
        p.out_lo = p.in_lo;
        p.out_hi = p.in_hi;
    }
}

// YkFDKBpPrecompute.cu:104-122 (L^2 expansion, 1/|SDD_plane|) and
// YkBpFdkKernel.cu:363 (voxel volume over the pixel area of the first view)
void build_pseudo_coefficients(const std::vector<FdkDerived>& g, const ykb_volume& vol,
    std::vector<PseudoViewCoef>& out)
{
    out.assign(g.size(), PseudoViewCoef{});
    if (g.empty()) return;
    const double cell = static_cast<double>(vol.vox_x) * vol.vox_y * vol.vox_z / (g[0].du * g[0].dv);
    for (size_t i = 0; i < g.size(); ++i) {
        const FdkDerived& d = g[i];
        const dvec3 r0 = dsub(d.detS, d.src);
        PseudoViewCoef& c = out[i];
        c.src[0] = d.src.x; c.src[1] = d.src.y; c.src[2] = d.src.z;
        c.l2[0] = static_cast<float>(ddot(r0, r0));
        c.l2[1] = static_cast<float>(2.0 * ddot(r0, d.detU));
        c.l2[2] = static_cast<float>(2.0 * ddot(r0, d.detV));
        c.l2[3] = static_cast<float>(ddot(d.detU, d.detU));
        c.l2[4] = static_cast<float>(2.0 * ddot(d.detU, d.detV));
        c.l2[5] = static_cast<float>(ddot(d.detV, d.detV));
        c.k = std::fabs(d.plane) > 1e-12 ? static_cast<float>(cell / std::fabs(d.plane)) : 0.f;
        c.ks = static_cast<float>(cell * std::fabs(d.plane));
    }
}

namespace {
double bessel_i0(double x)
{
    const double q = 0.25 * x * x;
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 500; ++k) {
        term *= q / (static_cast<double>(k) * k);
        sum += term;
        if (term < 1e-17 * sum) break;
    }
    return sum;
}

// Window shapes of src/Filter/YkCreateFilterKernelHelpers.cuh:38-103 in FP64.
double window_shape(double x, const ykb_filter& f)
{
    x = std::min(std::max(x, 0.0), 1.0);
    switch (f.type) {
    case 2: { const double t = 0.5 * kPi * x; return std::fabs(t) < 1e-8 ? 1.0 : std::sin(t) / t; }
    case 3: return std::cos(0.5 * kPi * x);
    case 4: return 0.5 * (1.0 + std::cos(kPi * x));
    case 5: return 0.54 + 0.46 * std::cos(kPi * x);
    case 6: return 0.42 + 0.5 * std::cos(kPi * x) + 0.08 * std::cos(2.0 * kPi * x);
    case 7: { const double o = std::max(static_cast<double>(f.butterworth_order), 0.01);
        return 1.0 / (1.0 + std::pow(x, 2.0 * o)); }
    case 8: { const double b = std::max(static_cast<double>(f.kaiser_beta), 0.0);
        const double t = 2.0 * x - 1.0;
        return bessel_i0(b * std::sqrt(std::max(0.0, 1.0 - t * t))) / bessel_i0(b); }
    case 9: { const double a = std::min(std::max(static_cast<double>(f.tukey_alpha), 0.0), 1.0);
        if (a <= 0.0) return 1.0;
        if (x < 0.5 * a) return 0.5 * (1.0 + std::cos(kPi * (2.0 * x / a - 1.0)));
        if (x <= 1.0 - 0.5 * a) return 1.0;
        return 0.5 * (1.0 + std::cos(kPi * (2.0 * x / a - 2.0 / a + 1.0))); }
    default: return 1.0;
    }
}
} // namespace

// Spatial kernel of the analytic frequency weights (AnalyticFreq of
// src/Filter/YkCreateFilterKernelKernels.cu:167-191, 1/N baked in, 1/du of
// src/Filter/YkCreateFilterKernelFFT.hpp:181-190; identity weights for
// EFdkFilter::None, :166-170): the inverse real DFT of length N = paddedN,
// h[d] for d in (-nu, nu).  Because N >= 2 nu, the reference's zero-padded
// circular convolution equals the linear Toeplitz product with these lags.
void build_ramp_kernel(int nu, double du, const ykb_filter& f, std::vector<double>& h)
{
    const int N = padded_fft_length(nu);
    const int nc = N / 2 + 1;
    std::vector<double> w(nc, 0.0);
    const double invN = 1.0 / N;
    if (f.type == 0) {
        for (int k = 0; k < nc; ++k) w[k] = static_cast<double>(f.gain) * invN;
    } else {
        const double cc = f.cutoff > 0.f ? static_cast<double>(f.cutoff) : 0.5;
        for (int k = 0; k < nc; ++k) {
            const double fr = static_cast<double>(k) / N;
            w[k] = fr > cc ? 0.0 : static_cast<double>(f.gain) * fr * window_shape(fr / cc, f) * invN / du;
        }
    }
    h.assign(2 * nu - 1, 0.0);
    std::vector<double> cosv(N);
    for (int k = 0; k < N; ++k) cosv[k] = std::cos(2.0 * kPi * k / N);
    for (int d = 0; d < nu; ++d) {
        double s = w[0];
        for (int k = 1; k < N / 2; ++k) {
            const long idx = (static_cast<long>(k) * d) % N;
            s += 2.0 * w[k] * cosv[idx];
        }
        s += w[N / 2] * ((d & 1) ? -1.0 : 1.0);
        h[nu - 1 + d] = s;
        h[nu - 1 - d] = s;
    }
}

// Joseph per-view data: normalizeToVoxel (src/common/cuda/operators/
// YkOperatorKernelTypes.cuh:148-168) in FP64, and the main axis decided in
// float on the centre ray of deriveProjectionFrame
// (include/YKCBCT/geometry/YkProjectionGeometry.hpp:114-147) with the
// tie-breaking of mainAxis (YkOperatorKernelTypes.cuh:133-141).
bool build_joseph_views(const ykb_cone_view* views, int n, int nu, int nv,
    const ykb_volume& vol, std::vector<JosephView>& out, std::string& why)
{
    if (n <= 0 || nu <= 0 || nv <= 0) { why = "empty view sequence or detector"; return false; }
    out.assign(n, JosephView{});
    const double ix = 1.0 / vol.vox_x, iy = 1.0 / vol.vox_y, iz = 1.0 / vol.vox_z;
    const int dims[3] = {vol.nx, vol.ny, vol.nz};
    const double vs[3] = {vol.vox_x, vol.vox_y, vol.vox_z};
    static const int perm[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
    for (int i = 0; i < n; ++i) {
        const ykb_cone_view& v = views[i];
        if (!finite4(v.src) || !finite4(v.detS) || !finite4(v.detU) || !finite4(v.detV)) {
            why = "non-finite view geometry";
            return false;
        }
        const float cu = 0.5f * static_cast<float>(nu - 1);
        const float cv = 0.5f * static_cast<float>(nv - 1);
        const float cx = v.detS.x + cu * v.detU.x + cv * v.detV.x;
        const float cy = v.detS.y + cu * v.detU.y + cv * v.detV.y;
        const float cz = v.detS.z + cu * v.detU.z + cv * v.detV.z;
        const float dx = cx - v.src.x, dy = cy - v.src.y, dz = cz - v.src.z;
        const float l2 = dx * dx + dy * dy + dz * dz;
        if (!std::isfinite(l2) || l2 <= 1e-12f) { why = "degenerate centre ray"; return false; }
        const float inv = 1.f / std::sqrt(l2);
        const float ax = std::fabs(dx * inv), ay = std::fabs(dy * inv), az = std::fabs(dz * inv);
        JosephView& j = out[i];
        j.axis = (ax >= ay && ax >= az) ? 0 : (ay >= ax && ay >= az) ? 1 : 2;
        j.src[0] = (v.src.x - static_cast<double>(vol.center_x)) * ix;
        j.src[1] = (v.src.y - static_cast<double>(vol.center_y)) * iy;
        j.src[2] = (v.src.z - static_cast<double>(vol.center_z)) * iz;
        j.detS[0] = (v.detS.x - static_cast<double>(vol.center_x)) * ix;
        j.detS[1] = (v.detS.y - static_cast<double>(vol.center_y)) * iy;
        j.detS[2] = (v.detS.z - static_cast<double>(vol.center_z)) * iz;
        j.detU[0] = v.detU.x * ix; j.detU[1] = v.detU.y * iy; j.detU[2] = v.detU.z * iz;
        j.detV[0] = v.detV.x * ix; j.detV[1] = v.detV.y * iy; j.detV[2] = v.detV.z * iz;
        j.n0 = dims[perm[j.axis][0]]; j.n1 = dims[perm[j.axis][1]]; j.n2 = dims[perm[j.axis][2]];
        j.v0 = vs[perm[j.axis][0]]; j.v1 = vs[perm[j.axis][1]]; j.v2 = vs[perm[j.axis][2]];
    }
    return true;
}

} // namespace ykb
