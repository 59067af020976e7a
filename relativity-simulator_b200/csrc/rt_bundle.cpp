// rt_bundle.cpp -- per-camera constants of the tracer (host, FP64).
//
// Everything here is computed once per camera; the per-pixel work runs on the
// device.  Citations are to the reference source tree.
#include <algorithm>
#include <cmath>

#include "rt_internal.h"

namespace relsim {

static double clampd(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
static double maxd(double a, double b) { return (a < b) ? b : a; }

// Bardeen-Press-Teukolsky ISCO, prograde for a >= 0
// (software_compute_engine.hpp:1052-1061).
double kerr_isco_radius(double m, double a_spin) {
    const double a_star = clampd(a_spin / maxd(m, 1e-12), -0.9999999, 0.9999999);
    const double abs_a = std::fabs(a_star);
    const double orbit_sign = (a_star >= 0.0) ? -1.0 : 1.0;
    const double cbrt_term = std::cbrt(maxd(1.0 - abs_a * abs_a, 0.0));
    const double z1 = 1.0 + cbrt_term * (std::cbrt(1.0 + abs_a) + std::cbrt(1.0 - abs_a));
    const double z2 = std::sqrt(3.0 * abs_a * abs_a + z1 * z1);
    return (3.0 + z2 + orbit_sign * std::sqrt(maxd((3.0 - z1) * (3.0 + z1 + 2.0 * z2), 0.0))) * m;
}

void build_bundle(const rt_camera& cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                  uint64_t ray_begin, uint64_t out_offset, BundleDesc& b) {
    b = BundleDesc{};
    b.ray_begin = ray_begin;
    b.out_offset = out_offset;
    b.width = cam.screen_width;
    b.height = cam.screen_height;
    b.col0 = col0;
    b.ncols = ncols;
    b.row0 = row0;
    b.nrows = nrows;
    b.max_steps = cam.max_integration_steps;

    // mass, spin clamp and outer horizon (software_compute_engine.hpp:3800-3803, 3370)
    const double m = maxd(cam.metric_mass, 1e-4);
    const double a = clampd(cam.metric_spin, -0.999 * m, 0.999 * m);
    const double rh = m + std::sqrt(maxd(m * m - a * a, 0.0));
    b.m = m;
    b.a = a;
    b.rh = rh;

    // observer (software_compute_engine.hpp:3902-3904)
    const double pi = 3.14159265358979323846;
    const double r_obs = maxd(cam.observer_position[1], rh * 1.02);
    const double th = clampd(cam.observer_position[2], 0.001, pi - 0.001);
    const double ph = cam.observer_position[3];
    b.st = std::sin(th);
    b.ct = std::cos(th);
    b.sp = std::sin(ph);
    b.cp = std::cos(ph);
    b.aspect = static_cast<double>(cam.screen_width) / static_cast<double>(cam.screen_height);
    b.tan_half_fov = std::tan(cam.field_of_view_rad * 0.5);  // camera_projections.hpp:33
    for (int i = 0; i < 3; ++i) {
        b.fwd[i] = cam.tetrad_e1[1 + i];
        b.rgt[i] = cam.tetrad_e2[1 + i];
        b.up[i] = cam.tetrad_e3[1 + i];
    }

    // observer KS position (kerr_schild_null_integrator.hpp:47-54)
    b.x0[0] = (r_obs * std::cos(ph) - a * std::sin(ph)) * std::sin(th);
    b.x0[1] = (r_obs * std::sin(ph) + a * std::cos(ph)) * std::sin(th);
    b.x0[2] = r_obs * std::cos(th);

    // field at x0 (kerr_schild_null_integrator.hpp:31-44)
    const double* x = b.x0;
    const double a2 = a * a, z2 = x[2] * x[2];
    const double diff = x[0] * x[0] + x[1] * x[1] + z2 - a2;
    const double r2 = maxd(0.5 * (diff + std::sqrt(diff * diff + 4.0 * a2 * z2)), 1e-24);
    const double r = std::sqrt(r2);
    const double hf = m * r2 * r / (r2 * r2 + a2 * z2);
    const double rpa = r2 + a2;
    const double k[3] = {(r * x[0] + a * x[1]) / rpa, (r * x[1] - a * x[0]) / rpa, x[2] / r};
    const double two_h = 2.0 * hf;
    b.two_h = two_h;
    for (int i = 0; i < 3; ++i) b.kf[i] = k[i];

    // static-observer tetrad by Gram-Schmidt under g = eta + 2H l l
    // (kerr_schild_null_integrator.hpp:154-177)
    auto inner = [&](const double* A, const double* B) {
        const double la = A[0] + k[0] * A[1] + k[1] * A[2] + k[2] * A[3];
        const double lb = B[0] + k[0] * B[1] + k[1] * B[2] + k[2] * B[3];
        return -A[0] * B[0] + A[1] * B[1] + A[2] * B[2] + A[3] * B[3] + two_h * la * lb;
    };
    const double u0 = 1.0 / std::sqrt(maxd(1.0 - two_h, 1e-6));
    b.u0 = u0;
    for (int i = 0; i < 3; ++i) {
        b.e[i][0] = two_h * k[i] * u0 * u0;
        b.e[i][1] = b.e[i][2] = b.e[i][3] = 0.0;
        b.e[i][1 + i] = 1.0;
    }
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < i; ++j) {
            const double proj = inner(b.e[i], b.e[j]);
            for (int c = 0; c < 4; ++c) b.e[i][c] -= proj * b.e[j][c];
        }
        const double inv_norm = 1.0 / std::sqrt(maxd(inner(b.e[i], b.e[i]), 1e-30));
        for (int c = 0; c < 4; ++c) b.e[i][c] *= inv_norm;
    }

    // unwrapped azimuth at the observer (kerr_schild_null_integrator.hpp:61-63)
    {
        const double raw = std::atan2(x[1], x[0]) - std::atan2(a, r);
        const double two_pi = 2.0 * pi;
        double d = raw - ph;
        d -= two_pi * std::floor(d / two_pi + 0.5);
        b.phi_start = ph + d;
        b.raw_phi0 = raw;
        b.wind0 = static_cast<int32_t>(std::lround((b.phi_start - raw) / two_pi));
    }

    // classification and integration
    b.r_capture = cam.capture_scale * rh;
    b.r_esc = cam.escape_radius;
    const bool disk = cam.disk_outer_radius > 0.0;
    b.r_in = (cam.disk_inner_radius > 0.0) ? cam.disk_inner_radius : kerr_isco_radius(m, a);
    b.r_out = cam.disk_outer_radius;
    b.r_early = disk ? b.r_in : 1e300;
    b.rtol = cam.rtol;
    b.atol = cam.atol;
    b.cap_c = cam.step_cap_fraction;
    b.h0 = cam.initial_step_fraction * r_obs;
    b.proj_tol = cam.projection_tol;
    b.fp64_radius = (cam.mixed_fp64_radius > 0.0) ? cam.mixed_fp64_radius : std::max(3.0 * rh, 5.0 * m);
    b.critical_band = (cam.mixed_critical_band < 0.0)   ? 0.0f
                      : (cam.mixed_critical_band > 0.0) ? static_cast<float>(cam.mixed_critical_band)
                                                        : kDefaultCriticalBand;
    b.flags = (disk ? BF_DISK : 0u) | (cam.early_capture ? BF_EARLY_CAPTURE : 0u) |
              (cam.precision_mode == RT_PRECISION_MIXED ? BF_MIXED : 0u);
}

double kn_horizon(double m, double a, double q) {
    const double diff = m * m - a * a - q * q;  // kerr_newman.hpp:95-101
    return (diff < 0.0) ? m : m + std::sqrt(diff);
}

// Boyer-Lindquist Kerr-Newman camera (trace_exact_photon_dispatch,
// software_compute_engine.hpp:3364-3368 and :3388-3391): r_+ of the
// Kerr-Newman metric, ISCO and disk from the Kerr formula, and the ZAMO tetrad
// at the observer (observer_tetrad.hpp:82-100): omega = -g_tphi / g_phiphi,
// alpha^2 = -(g_tt + omega g_tphi), e0 = (1, 0, 0, omega) / alpha and the unit
// coordinate vectors (orthonormal already; the reference's Gram-Schmidt pass
// moves them only by rounding).
void build_bl_bundle(const rt_camera& cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                     uint64_t ray_begin, uint64_t out_offset, BlDesc& b) {
    b = BlDesc{};
    b.ray_begin = ray_begin;
    b.out_offset = out_offset;
    b.width = cam.screen_width;
    b.height = cam.screen_height;
    b.col0 = col0;
    b.ncols = ncols;
    b.row0 = row0;
    b.nrows = nrows;
    b.max_steps = cam.max_integration_steps;

    const double m = maxd(cam.metric_mass, 1e-4);
    const double a = clampd(cam.metric_spin, -0.999 * m, 0.999 * m);
    const double q = cam.metric_charge;
    const double rh = kn_horizon(m, a, q);
    b.m = m;
    b.a = a;
    b.q2 = q * q;
    b.rh = rh;

    const double pi = 3.14159265358979323846;
    const double r_obs = maxd(cam.observer_position[1], rh * 1.02);
    const double th = clampd(cam.observer_position[2], 0.001, pi - 0.001);
    const double ph = cam.observer_position[3];
    b.r_obs = r_obs;
    b.th_obs = th;
    b.ph_obs = ph;
    b.st = std::sin(th);
    b.ct = std::cos(th);
    b.sp = std::sin(ph);
    b.cp = std::cos(ph);
    b.aspect = static_cast<double>(cam.screen_width) / static_cast<double>(cam.screen_height);
    b.tan_half_fov = std::tan(cam.field_of_view_rad * 0.5);
    for (int i = 0; i < 3; ++i) {
        b.fwd[i] = cam.tetrad_e1[1 + i];
        b.rgt[i] = cam.tetrad_e2[1 + i];
        b.up[i] = cam.tetrad_e3[1 + i];
    }

    // metric at the observer (kerr_newman.hpp:141-169)
    const double s = std::sin(th), c = std::cos(th);
    const double s2 = s * s, a2 = a * a, r2 = r_obs * r_obs;
    const double rho2 = r2 + a2 * c * c;
    const double delta = r2 - 2.0 * m * r_obs + a2 + b.q2;
    const double F = (2.0 * m * r_obs - b.q2) / rho2;
    const double g_tt = F - 1.0, g_tp = -a * s2 * F, g_rr = rho2 / delta, g_thth = rho2;
    const double g_pp = s2 * (r2 + a2 + a2 * s2 * F);
    const double omega = -g_tp / g_pp;
    const double alpha = std::sqrt(maxd(-(g_tt + omega * g_tp), 1e-30));
    b.e0_t = 1.0 / alpha;
    b.e0_phi = omega / alpha;
    b.e_r = 1.0 / std::sqrt(maxd(g_rr, 1e-30));
    b.e_th = 1.0 / std::sqrt(maxd(g_thth, 1e-30));
    b.e_ph = 1.0 / std::sqrt(maxd(g_pp, 1e-30));

    b.r_capture = cam.capture_scale * rh;
    b.r_esc = cam.escape_radius;
    const bool disk = cam.disk_outer_radius > 0.0;
    b.r_in = (cam.disk_inner_radius > 0.0) ? cam.disk_inner_radius : kerr_isco_radius(m, a);
    b.r_out = cam.disk_outer_radius;
    b.r_early = disk ? b.r_in : 1e300;
    b.rtol = cam.rtol;
    b.atol = cam.atol;
    b.cap_c = cam.step_cap_fraction;
    b.h0 = cam.initial_step_fraction * r_obs;
    b.proj_tol = cam.projection_tol;
    b.flags = (disk ? BF_DISK : 0u) | (cam.early_capture ? BF_EARLY_CAPTURE : 0u);
}

// Source table of a multi-source scene (software_compute_engine.hpp:2738-2798):
// the camera's hole at the origin, then each body with its spin axis
// normalised and a local frame from a helper axis (z unless the spin axis is
// near z, then x).  The camera's disk radii are absolute (inner <= 0: r_ISCO),
// a body's are scaled as in the reference.
uint32_t build_ms_sources(const rt_camera& cam, const rt_source* src, uint32_t n, MsSource* out) {
    const double m = maxd(cam.metric_mass, 1e-4);
    const double a = clampd(cam.metric_spin, -0.999 * m, 0.999 * m);
    const double rh = m + std::sqrt(maxd(m * m - a * a, 0.0));
    MsSource p{};
    p.m = m;
    p.a = a;
    p.axis[2] = 1.0;
    p.fx[0] = 1.0;
    p.fy[1] = 1.0;
    p.rh = rh;
    p.req = std::sqrt(rh * rh + a * a);
    if (cam.disk_outer_radius > 0.0) {
        p.disk_in = (cam.disk_inner_radius > 0.0) ? cam.disk_inner_radius : kerr_isco_radius(m, a);
        p.disk_out = cam.disk_outer_radius;
    } else {
        p.disk_in = p.disk_out = -1.0;
    }
    out[0] = p;
    uint32_t count = 1;
    for (uint32_t b = 0; b < n && count < kMaxSources; ++b) {
        const rt_source& s = src[b];
        MsSource q{};
        const double mb = maxd(s.mass, 1e-9);
        const double ab = clampd(s.spin_parameter, -0.9999, 0.9999) * mb;
        const double rhb = mb + std::sqrt(maxd(mb * mb - ab * ab, 0.0));
        const double len = std::sqrt(s.axis[0] * s.axis[0] + s.axis[1] * s.axis[1] + s.axis[2] * s.axis[2]);
        double ax[3] = {0.0, 0.0, 1.0};
        if (len > 1e-12)
            for (int k = 0; k < 3; ++k) ax[k] = s.axis[k] / len;
        const bool near_z = !(std::fabs(ax[2]) < 0.9);
        const double hp[3] = {near_z ? 1.0 : 0.0, 0.0, near_z ? 0.0 : 1.0};
        double fx[3] = {hp[1] * ax[2] - hp[2] * ax[1], hp[2] * ax[0] - hp[0] * ax[2], hp[0] * ax[1] - hp[1] * ax[0]};
        const double fl = std::sqrt(fx[0] * fx[0] + fx[1] * fx[1] + fx[2] * fx[2]);
        for (double& v : fx) v /= fl;
        const double fy[3] = {ax[1] * fx[2] - ax[2] * fx[1], ax[2] * fx[0] - ax[0] * fx[2],
                              ax[0] * fx[1] - ax[1] * fx[0]};
        for (int k = 0; k < 3; ++k) {
            q.pos[k] = s.position[k];
            q.axis[k] = ax[k];
            q.fx[k] = fx[k];
            q.fy[k] = fy[k];
        }
        q.m = mb;
        q.a = ab;
        q.rh = rhb;
        q.req = std::sqrt(rhb * rhb + ab * ab);
        if (s.disk_enabled > 0.5) {
            const double inner = kerr_isco_radius(mb, ab) * maxd(s.disk_inner_scale, 1.0);
            q.disk_in = inner;
            q.disk_out = maxd(s.disk_outer_units * mb, inner * 1.05);
        } else {
            q.disk_in = q.disk_out = -1.0;
        }
        out[count++] = q;
    }
    return count;
}

// Per-camera constants of a multi-source bundle: the observer at the Cartesian
// point of (r, theta, phi) and the tetrad directions (trace_multi_source,
// software_compute_engine.hpp:3049-3068).
void build_ms_bundle(const rt_camera& cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                     uint64_t ray_begin, uint64_t out_offset, uint32_t src_begin, uint32_t src_count, MsDesc& b) {
    b = MsDesc{};
    b.ray_begin = ray_begin;
    b.out_offset = out_offset;
    b.width = cam.screen_width;
    b.height = cam.screen_height;
    b.col0 = col0;
    b.ncols = ncols;
    b.row0 = row0;
    b.nrows = nrows;
    b.max_steps = cam.max_integration_steps;
    b.src_begin = src_begin;
    b.src_count = src_count;
    const double pi = 3.14159265358979323846;
    const double r = cam.observer_position[1];
    const double th = clampd(cam.observer_position[2], 0.001, pi - 0.001);
    const double ph = cam.observer_position[3];
    b.x0[0] = r * std::sin(th) * std::cos(ph);
    b.x0[1] = r * std::sin(th) * std::sin(ph);
    b.x0[2] = r * std::cos(th);
    b.phi0 = std::atan2(b.x0[1], b.x0[0]);
    b.aspect = static_cast<double>(cam.screen_width) / static_cast<double>(cam.screen_height);
    b.tan_half_fov = std::tan(cam.field_of_view_rad * 0.5);
    for (int i = 0; i < 3; ++i) {
        b.fwd[i] = cam.tetrad_e1[1 + i];
        b.rgt[i] = cam.tetrad_e2[1 + i];
        b.up[i] = cam.tetrad_e3[1 + i];
    }
    b.rtol = cam.rtol;
    b.atol = cam.atol;
    b.cap_c = cam.step_cap_fraction;
    b.h0 = cam.initial_step_fraction * r;
    b.proj_tol = cam.projection_tol;
    b.r_esc = cam.escape_radius;
    b.capture_scale = cam.capture_scale;
}

void row_window(const rt_camera& c, uint32_t& row0, uint32_t& nrows) {
    row0 = std::min(c.dispatch_row_offset, c.screen_height);
    nrows = (c.dispatch_row_count == 0) ? (c.screen_height - row0)
                                        : std::min(c.dispatch_row_count, c.screen_height - row0);
}

}  // namespace relsim
