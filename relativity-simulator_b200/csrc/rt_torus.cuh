// rt_torus.cuh -- the Fishbone-Moncrief torus of hydro model 2 as host/device
// code: the constant-angular-momentum equilibrium torus around a Kerr hole
// (Fishbone & Moncrief 1976), as hydro/fishbone_moncrief.hpp states it with
// G = c = 1, and the bounds that render/accretion_disk/hydro_disk_shading.hpp
// (:76-110) draws around it.  The shading of a chord through the torus is
// fm_segment in rt_shade.cuh.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define RT_FM_HD __host__ __device__ inline
#else
#define RT_FM_HD inline
#endif

namespace relsim {
namespace torus {

// The torus's hole and constants: mass m, spin a (clamped to 0.999 m), outer
// horizon rh, specific angular momentum l (Keplerian at the pressure maximum)
// and the potential w_in at the inner edge.
struct Torus {
    double m, a, rh, l, w_in;
};

RT_FM_HD double fmx(double a, double b) { return (a < b) ? b : a; }

RT_FM_HD double horizon(double m, double a) {
    const double d = m * m - a * a;
    return (d < 0.0) ? m : m + sqrt(d);
}

// Keplerian specific angular momentum at radius r (fishbone_moncrief.hpp:98-116).
RT_FM_HD double keplerian_l(double m, double a, double rh, double r) {
    const double rs = fmx(r, 1.001 * rh);
    const double sm = sqrt(m), sr = sqrt(rs);
    const double num = sm * (rs * rs - 2.0 * a * sm * sr + a * a);
    const double den = rs * sr - 2.0 * m * sr + a * sm;
    return (fabs(den) < 1e-30) ? 0.0 : num / den;
}

// Potential W = ln(-u_t) of the torus's fluid at (r, theta) in Boyer-Lindquist
// coordinates (:118-150); 1e30 where no such orbit exists.
RT_FM_HD double potential(double m, double a, double rh, double l, double r, double theta) {
    if (r <= rh * 1.0001) return 1e30;
    const double st = sin(theta), ct = cos(theta);
    const double s2 = fmx(st * st, 1e-30), c2 = ct * ct;
    const double r2 = r * r, a2 = a * a;
    const double rho2 = r2 + a2 * c2;
    const double delta = r2 - 2.0 * m * r + a2;
    const double sigma = (r2 + a2) * (r2 + a2) - a2 * delta * s2;
    const double denom = sigma * s2 - 4.0 * m * r * a * l * s2 - l * l * (delta - a2 * s2);
    if (denom <= 0.0 || delta <= 0.0) return 1e30;
    return 0.5 * log(fmx((rho2 * delta * s2) / denom, 1e-30));
}
RT_FM_HD double potential(const Torus& t, double r, double theta) { return potential(t.m, t.a, t.rh, t.l, r, theta); }

// Specific enthalpy h = exp(W_in - W), at least 1 (:152-159).
RT_FM_HD double enthalpy(const Torus& t, double r, double theta) {
    const double w = potential(t, r, theta);
    if (w >= t.w_in) return 1.0;
    return fmx(1.0, exp(t.w_in - w));
}

// The fluid's u^t and u^phi (:210-224): u_t = -e^W, u_phi = -l u_t, raised
// with the Boyer-Lindquist Kerr inverse metric (metrics/kerr.hpp:151-177).
RT_FM_HD void four_velocity(const Torus& t, double r, double theta, double& ut, double& uphi) {
    const double w = potential(t, r, theta);
    if (w >= 1e20) {
        ut = 1.0;
        uphi = 0.0;
        return;
    }
    const double lt = -exp(w), lphi = -t.l * lt;
    const double rr = fmx(r, 1e-12);
    const double st = sin(theta), ct = cos(theta);
    const double s2 = fmx(st * st, 1e-30), c2 = ct * ct;
    const double a2 = t.a * t.a, r2 = rr * rr;
    const double rho2 = r2 + a2 * c2;
    const double delta = r2 - 2.0 * t.m * rr + a2;
    const double sigma = (r2 + a2) * (r2 + a2) - a2 * delta * s2;
    const double gtt = -sigma / (rho2 * delta);
    const double gtp = -(2.0 * t.m * rr * t.a) / (rho2 * delta);
    const double gpp = (delta - a2 * s2) / (rho2 * delta * s2);
    ut = gtt * lt + gtp * lphi;
    uphi = gtp * lt + gpp * lphi;
}

// The torus of a hole (mass, spin clamped as the shading context does) with its
// inner edge and pressure maximum at r_in and r_center (units of M; 6 and 12
// when not positive): the constants, the peak enthalpy and the radial bounds
// the shading samples within (0.8 r_in, and 1.05 times the equatorial outer
// edge found by a scan in steps of r_center / 4 and 48 bisections; 200
// r_center when the torus does not close).  valid: a torus with h_max > 1.
struct TorusContext {
    Torus t;
    double h_max, inner_bound, outer_bound;
    bool valid, closed;
};

RT_FM_HD TorusContext make_torus(double mass, double spin, double r_in_units, double r_center_units) {
    TorusContext c{};
    const double m = fmx(mass, 1e-9);
    const double lim = 0.999 * m;
    const double a = (spin < -lim) ? -lim : ((lim < spin) ? lim : spin);
    const double rh = horizon(m, a);
    const double r_c = (r_center_units * m > 0.0) ? r_center_units * m : 12.0 * m;
    const double r_in = (r_in_units * m > 0.0) ? r_in_units * m : 6.0 * m;
    const double half_pi = 1.57079632679489661923;
    c.t = Torus{m, a, rh, keplerian_l(m, a, rh, r_c), 0.0};
    c.t.w_in = potential(c.t, r_in, half_pi);
    const double w_center = potential(c.t, r_c, half_pi);
    c.h_max = exp(fmx(0.0, c.t.w_in - w_center));
    c.valid = std::isfinite(c.h_max) && (c.h_max > 1.0 + 1e-9);
    c.inner_bound = 0.8 * r_in;
    c.outer_bound = 0.0;
    c.closed = false;
    if (!c.valid) return c;
    const double scan_step = 0.25 * r_c, scan_limit = 200.0 * r_c;
    double inside = r_c, outside = r_c;
    bool found = false;
    while (outside < scan_limit) {
        outside += scan_step;
        if (!(potential(c.t, outside, half_pi) < c.t.w_in)) {
            found = true;
            break;
        }
        inside = outside;
    }
    if (found) {
        for (int it = 0; it < 48; ++it) {
            const double mid = 0.5 * (inside + outside);
            if (potential(c.t, mid, half_pi) < c.t.w_in) inside = mid;
            else outside = mid;
        }
        c.outer_bound = 1.05 * outside;
    } else {
        c.outer_bound = scan_limit;
    }
    c.closed = found;
    return c;
}

}  // namespace torus
}  // namespace relsim
