/*
 * ks_oracle.c -- FP64 CPU oracle of the backward null-geodesic tracer.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  Every function
 * cites the reference file:line it restates; paths are relative to the
 * Wartets/Relativity-Simulator source tree.
 *
 * Integration scheme (FP64 DP45, composed from reference parts):
 *   state y = (x, y, z, p_x, p_y, p_z) in Kerr-Schild Cartesian coordinates with
 *   p_t = -1, integrated backwards (h < 0) with Dormand-Prince 5(4),
 *   PI30 control, FSAL reuse of the last stage, a constraint projection onto
 *   H = 0 after every accepted step and a step cap |h| <= c max(r - r_+, 0.01 M).
 */
#include "ks_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define ORC_PI 3.14159265358979323846

/* std::max / std::min / std::clamp semantics (NaN propagation included). */
static inline double max_d(double a, double b) { return (a < b) ? b : a; }
static inline double min_d(double a, double b) { return (b < a) ? b : a; }
static inline double clamp_d(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

typedef struct {
    double r, h, k[3];
} field_t;

/* kerr_schild_null_integrator.hpp:31-44 */
static field_t ks_field(const double* x, double mass, double spin)
{
    field_t f;
    const double a2 = spin * spin;
    const double z2 = x[2] * x[2];
    const double diff = x[0] * x[0] + x[1] * x[1] + z2 - a2;
    const double r2 = max_d(0.5 * (diff + sqrt(diff * diff + 4.0 * a2 * z2)), 1e-24);
    const double r = sqrt(r2);
    const double den = r2 * r2 + a2 * z2;
    const double rpa = r2 + a2;
    f.r = r;
    f.h = mass * r2 * r / den;
    f.k[0] = (r * x[0] + spin * x[1]) / rpa;
    f.k[1] = (r * x[1] - spin * x[0]) / rpa;
    f.k[2] = x[2] / r;
    return f;
}

/* kerr_schild_null_integrator.hpp:72-114.  Returns the BL radius of y. */
static double ks_rhs(const double* y, double mass, double spin, double* dy)
{
    const double* x = y;
    const double* p = y + 3;
    const field_t f = ks_field(x, mass, spin);
    const double r = f.r;
    const double r2 = r * r;
    const double r3 = r2 * r;
    const double r4 = r2 * r2;
    const double a2 = spin * spin;
    const double z2 = x[2] * x[2];
    const double den = r4 + a2 * z2;
    const double rpa = r2 + a2;
    const double inv_rpa2 = 1.0 / (rpa * rpa);
    const double inv_den2 = 1.0 / (den * den);
    const double s = f.k[0] * p[0] + f.k[1] * p[1] + f.k[2] * p[2] + 1.0;

    for (int i = 0; i < 3; ++i) dy[i] = p[i] - 2.0 * f.h * s * f.k[i];

    const double dr[3] = {r3 * x[0] / den, r3 * x[1] / den, r * rpa * x[2] / den};
    const double bracket = 3.0 * a2 * z2 - r4;
    const double nx = r * x[0] + spin * x[1];
    const double ny = r * x[1] - spin * x[0];
    for (int i = 0; i < 3; ++i) {
        double dh = mass * dr[i] * r2 * bracket * inv_den2;
        if (i == 2) dh -= 2.0 * mass * a2 * r3 * x[2] * inv_den2;
        const double ex = (i == 0) ? 1.0 : 0.0;
        const double ey = (i == 1) ? 1.0 : 0.0;
        const double ez = (i == 2) ? 1.0 : 0.0;
        const double dk1 = ((dr[i] * x[0] + r * ex + spin * ey) * rpa - nx * 2.0 * r * dr[i]) * inv_rpa2;
        const double dk2 = ((dr[i] * x[1] + r * ey - spin * ex) * rpa - ny * 2.0 * r * dr[i]) * inv_rpa2;
        const double dk3 = (r * ez - x[2] * dr[i]) / r2;
        const double dkp = dk1 * p[0] + dk2 * p[1] + dk3 * p[2];
        dy[3 + i] = dh * s * s + 2.0 * f.h * s * dkp;
    }
    return r;
}

void orc_ks_field(const double x[3], double mass, double spin, double* r, double* h, double k[3])
{
    const field_t f = ks_field(x, mass, spin);
    *r = f.r;
    *h = f.h;
    k[0] = f.k[0];
    k[1] = f.k[1];
    k[2] = f.k[2];
}

void orc_ks_rhs(const double y[6], double mass, double spin, double dy[6]) { (void)ks_rhs(y, mass, spin, dy); }

/* kerr_schild_null_integrator.hpp:47-54 */
void orc_ks_position_from_bl(double r, double theta, double phi, double spin, double out[3])
{
    const double st = sin(theta);
    out[0] = (r * cos(phi) - spin * sin(phi)) * st;
    out[1] = (r * sin(phi) + spin * cos(phi)) * st;
    out[2] = r * cos(theta);
}

/* kerr_schild_null_integrator.hpp:57-69: (r, theta, unwrapped phi). */
void orc_bl_from_ks(const double x[3], double spin, double previous_phi, double out[3])
{
    const field_t f = ks_field(x, 0.0, spin);
    const double rho = sqrt(max_d(f.r * f.r - x[2] * x[2], 0.0));
    const double two_pi = 2.0 * ORC_PI;
    const double raw_phi = atan2(x[1], x[0]) - atan2(spin, f.r);
    double delta = raw_phi - previous_phi;
    delta -= two_pi * floor(delta / two_pi + 0.5);
    out[0] = f.r;
    out[1] = atan2(rho, x[2]);
    out[2] = previous_phi + delta;
}

/* kerr_schild_null_integrator.hpp:142-194: static-observer tetrad (Gram-Schmidt
 * under g = eta + 2H l l) and the null covector with p_t = -1. */
void orc_initial_momentum(const double x[3], double mass, double spin, const double outward[3], double p[3])
{
    const field_t f = ks_field(x, mass, spin);
    const double two_h = 2.0 * f.h;
    const double* k = f.k;
#define ORC_INNER(A, B)                                                                    \
    (-(A)[0] * (B)[0] + (A)[1] * (B)[1] + (A)[2] * (B)[2] + (A)[3] * (B)[3] +              \
     two_h * ((A)[0] + k[0] * (A)[1] + k[1] * (A)[2] + k[2] * (A)[3]) *                   \
         ((B)[0] + k[0] * (B)[1] + k[1] * (B)[2] + k[2] * (B)[3]))
    const double u0 = 1.0 / sqrt(max_d(1.0 - two_h, 1e-6));
    double e[3][4];
    for (int i = 0; i < 3; ++i) {
        e[i][0] = two_h * k[i] * u0 * u0;
        e[i][1] = e[i][2] = e[i][3] = 0.0;
        e[i][1 + i] = 1.0;
    }
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < i; ++j) {
            const double proj = ORC_INNER(e[i], e[j]);
            for (int c = 0; c < 4; ++c) e[i][c] -= proj * e[j][c];
        }
        const double inv_norm = 1.0 / sqrt(max_d(ORC_INNER(e[i], e[i]), 1e-30));
        for (int c = 0; c < 4; ++c) e[i][c] *= inv_norm;
    }
#undef ORC_INNER
    double v[4] = {u0, 0.0, 0.0, 0.0};
    for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 4; ++c) v[c] -= outward[i] * e[i][c];
    const double lv = v[0] + k[0] * v[1] + k[1] * v[2] + k[2] * v[3];
    const double p_t = -v[0] + two_h * lv;
    const double inv_e = 1.0 / max_d(-p_t, 1e-12);
    p[0] = (v[1] + two_h * lv * k[0]) * inv_e;
    p[1] = (v[2] + two_h * lv * k[1]) * inv_e;
    p[2] = (v[3] + two_h * lv * k[2]) * inv_e;
}

/* software_compute_engine.hpp:1052-1061 (Bardeen-Press-Teukolsky ISCO). */
double orc_isco_radius(double m, double a_spin)
{
    const double a_star = clamp_d(a_spin / max_d(m, 1e-12), -0.9999999, 0.9999999);
    const double abs_a = fabs(a_star);
    const double orbit_sign = (a_star >= 0.0) ? -1.0 : 1.0;
    const double cbrt_term = cbrt(max_d(1.0 - abs_a * abs_a, 0.0));
    const double z1 = 1.0 + cbrt_term * (cbrt(1.0 + abs_a) + cbrt(1.0 - abs_a));
    const double z2 = sqrt(3.0 * abs_a * abs_a + z1 * z1);
    const double r = 3.0 + z2 + orbit_sign * sqrt(max_d((3.0 - z1) * (3.0 + z1 + 2.0 * z2), 0.0));
    return r * m;
}

/* accretion_disk_model.hpp:205-225: circular-orbit frame and g. */
double orc_redshift_at(double mass, double spin, double radius, double lz)
{
    const double spin_mag = fabs(spin);
    const double sqrt_m = sqrt(max_d(mass, 1e-12));
    const double sqrt_r = sqrt(max_d(radius, 1e-12));
    const double r15 = radius * sqrt_r;
    const double angular = sqrt_m / (r15 + spin_mag * sqrt_m);
    const double bracket = max_d(r15 - 3.0 * mass * sqrt_r + 2.0 * spin_mag * sqrt_m, 1e-9);
    const double omega = (spin < 0.0) ? -angular : angular;
    const double ut = (r15 + spin_mag * sqrt_m) / (sqrt(r15) * sqrt(bracket));
    const double den = ut * (1.0 - omega * lz);
    return (fabs(den) > 1e-9) ? clamp_d(1.0 / den, 0.05, 4.0) : 1.0;
}

/* camera_projections.hpp:27-40 */
void orc_pinhole_ray(double u, double v, double fov, double n[3])
{
    const double t = tan(fov * 0.5);
    const double n1 = 1.0, n2 = v * t, n3 = u * t;
    const double len = sqrt(n1 * n1 + n2 * n2 + n3 * n3);
    const double inv = (len > 0.0) ? (1.0 / len) : 1.0;
    n[0] = n1 * inv;
    n[1] = n2 * inv;
    n[2] = n3 * inv;
}

/* step_controller.hpp:44-78 (PI30 branch), written as exp/log of the same
 * exponents: factor = (1/e)^(0.7/k) (e_prev/e)^(0.3/k). */
static inline double pi30(double le, double lp, double order_p1)
{
    return exp(-(0.7 / order_p1) * le + (0.3 / order_p1) * (lp - le));
}

double orc_pi30_factor(double err, double err_prev, int has_history, double order_p1)
{
    const double safe_err = max_d(err, 1e-12);
    const double safe_prev = has_history ? max_d(err_prev, 1e-12) : safe_err;
    return pi30(log(safe_err), log(safe_prev), order_p1);
}

/* H = 1/2 (|p|^2 - 1 - 2 H_f s^2), the Hamiltonian of g^{mu nu} = eta - 2 H_f l l
 * (kerr_schild.hpp:168-189) evaluated with p_t = -1. */
double orc_hamiltonian(const double y[6], double mass, double spin)
{
    const field_t f = ks_field(y, mass, spin);
    const double* p = y + 3;
    const double s = 1.0 + f.k[0] * p[0] + f.k[1] * p[1] + f.k[2] * p[2];
    return 0.5 * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] - 1.0 - 2.0 * f.h * s * s);
}

/* E = -p_t recovered from the null condition at fixed p_i. */
static double energy_from_null(const double y[6], double mass, double spin)
{
    const field_t f = ks_field(y, mass, spin);
    const double* p = y + 3;
    const double kp = f.k[0] * p[0] + f.k[1] * p[1] + f.k[2] * p[2];
    const double pp = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    const double a = 1.0 + 2.0 * f.h;
    const double b = 2.0 * f.h * kp; /* half of the linear coefficient */
    const double c = pp - 2.0 * f.h * kp * kp;
    return (-b + sqrt(max_d(b * b + a * c, 0.0))) / a;
}

/* Carter constant with E = 1 and mu = 0 (kerr_invariants.hpp:45-48); BL p_theta
 * is the KS covector contracted with dx^i/dtheta of the map at
 * kerr_schild_null_integrator.hpp:47-53. */
double orc_carter_q(const double y[6], double mass, double spin)
{
    const field_t f = ks_field(y, mass, spin);
    const double* x = y;
    const double* p = y + 3;
    const double r = f.r;
    const double cos_t = clamp_d(x[2] / r, -1.0, 1.0);
    const double sin2 = max_d((x[0] * x[0] + x[1] * x[1]) / (r * r + spin * spin), 1e-30);
    const double sin_t = sqrt(sin2);
    const double p_theta = (x[0] * p[0] + x[1] * p[1]) * cos_t / sin_t - r * sin_t * p[2];
    const double lz = x[0] * p[1] - x[1] * p[0];
    return p_theta * p_theta + cos_t * cos_t * (-spin * spin + lz * lz / sin2);
}

/* Signed distance (in impact parameter, units of M) of the constants (xi, eta)
 * from the Kerr critical curve: the local minimum R_min of the radial quartic
 * R(r) = r^4 + P r^2 + Qc r - a^2 eta (carter_ray_classifier.hpp:132-135) outside
 * r_+ is pushed to zero by d_eta = R_min / Delta(r*), and d_b = d_eta / (2 b).
 * Positive: no turning point (captured side). */
double orc_shadow_distance(double mass, double spin, double xi, double eta)
{
    const double a2 = spin * spin;
    const double P = a2 - xi * xi - eta;
    const double Qc = 2.0 * mass * (eta + (xi - spin) * (xi - spin));
    const double R0 = -a2 * eta;
    const double rp = mass + sqrt(max_d(mass * mass - a2, 0.0));
    /* R'(r) = 4 r^3 + 2 P r + Qc = 0  ->  t^3 + p t + q = 0 */
    const double pp = 0.5 * P, qq = 0.25 * Qc;
    double roots[3];
    int n = 0;
    const double disc = -(4.0 * pp * pp * pp + 27.0 * qq * qq);
    if (disc > 0.0 && pp < 0.0) {
        const double m2 = 2.0 * sqrt(-pp / 3.0);
        const double arg = clamp_d(3.0 * qq / (pp * m2), -1.0, 1.0);
        const double th = acos(arg) / 3.0;
        for (int k = 0; k < 3; ++k) roots[n++] = m2 * cos(th - 2.0 * ORC_PI * k / 3.0);
    } else {
        const double sq = sqrt(max_d(qq * qq / 4.0 + pp * pp * pp / 27.0, 0.0));
        roots[n++] = cbrt(-qq / 2.0 + sq) + cbrt(-qq / 2.0 - sq);
    }
    double best = INFINITY;
    double best_r = 0.0;
    for (int i = 0; i < n; ++i) {
        const double r = roots[i];
        if (!(r > rp)) continue;
        if (12.0 * r * r + 2.0 * P <= 0.0) continue; /* not a minimum */
        const double R = ((r * r + P) * r + Qc) * r + R0;
        if (R < best) {
            best = R;
            best_r = r;
        }
    }
    if (!isfinite(best)) return INFINITY;
    const double delta = best_r * best_r - 2.0 * mass * best_r + a2;
    const double b = sqrt(max_d(eta + xi * xi, 1e-30));
    return best / max_d(delta, 1e-30) / (2.0 * b);
}

/* ---------------------------------------------------------------------- */
/* Per-camera constants (software_compute_engine.hpp:3790-3803, 3902-3912). */
typedef struct {
    double m, a, rh;
    double r_obs, th_obs, ph_obs;
    double aspect, fov;
    double fwd[3], rgt[3], up[3];
    double r_in, r_out, r_capture, r_esc;
    int disk;
} cam_consts;

static void camera_consts(const orc_camera* cam, cam_consts* c)
{
    c->m = max_d(cam->metric_mass, 1e-4);
    c->a = clamp_d(cam->metric_spin, -0.999 * c->m, 0.999 * c->m);
    c->rh = c->m + sqrt(max_d(c->m * c->m - c->a * c->a, 0.0));
    c->r_obs = max_d(cam->observer_position[1], c->rh * 1.02);
    c->th_obs = clamp_d(cam->observer_position[2], 0.001, ORC_PI - 0.001);
    c->ph_obs = cam->observer_position[3];
    c->aspect = (double)cam->screen_width / (double)cam->screen_height;
    c->fov = cam->field_of_view_rad;
    for (int i = 0; i < 3; ++i) {
        c->fwd[i] = cam->tetrad_e1[1 + i];
        c->rgt[i] = cam->tetrad_e2[1 + i];
        c->up[i] = cam->tetrad_e3[1 + i];
    }
    c->r_in = (cam->disk_inner_radius > 0.0) ? cam->disk_inner_radius : orc_isco_radius(c->m, c->a);
    c->r_out = cam->disk_outer_radius;
    c->disk = cam->disk_outer_radius > 0.0;
    c->r_capture = cam->capture_scale * c->rh;
    c->r_esc = cam->escape_radius;
}

/* software_compute_engine.hpp:3843-3862 (pixel -> world direction),
 * :3912-3938 (spherical components) and :1637-1650 (KS state). */
static double initial_state(const orc_camera* cam, const cam_consts* c, uint32_t px, uint32_t py, double y0[6])
{
    const double W = (double)cam->screen_width, H = (double)cam->screen_height;
    const double v = 1.0 - ((double)py + 0.5) / H * 2.0;
    const double u = (((double)px + 0.5) / W * 2.0 - 1.0) * c->aspect;
    double n[3];
    orc_pinhole_ray(u, v, c->fov, n);
    double d[3];
    for (int i = 0; i < 3; ++i) d[i] = n[0] * c->fwd[i] + n[2] * c->rgt[i] + n[1] * c->up[i];
    const double st = sin(c->th_obs), ct = cos(c->th_obs), sp = sin(c->ph_obs), cp = cos(c->ph_obs);
    const double n_r = d[0] * (st * cp) + d[1] * (st * sp) + d[2] * ct;
    const double n_th = d[0] * (ct * cp) + d[1] * (ct * sp) + d[2] * (-st);
    const double n_ph = d[0] * (-sp) + d[1] * cp + d[2] * 0.0;
    const double outward[3] = {n_r * st * cp + n_th * ct * cp - n_ph * sp, n_r * st * sp + n_th * ct * sp + n_ph * cp,
                               n_r * ct - n_th * st};
    orc_ks_position_from_bl(c->r_obs, c->th_obs, c->ph_obs, c->a, y0);
    orc_initial_momentum(y0, c->m, c->a, outward, y0 + 3);
    return y0[0] * y0[4] - y0[1] * y0[3];
}

double orc_ray_initial_state(const orc_camera* cam, uint32_t px, uint32_t py, double y0[6])
{
    cam_consts c;
    camera_consts(cam, &c);
    return initial_state(cam, &c, px, py, y0);
}

/* Dormand-Prince 5(4) coefficients (rk45_adaptive.hpp:196-203). */
static const double A21 = 1.0 / 5.0;
static const double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
static const double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
static const double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0, A54 = -212.0 / 729.0;
static const double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0, A64 = 49.0 / 176.0,
                    A65 = -5103.0 / 18656.0;
static const double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0, B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
static const double E1 = 71.0 / 57600.0, E3 = -71.0 / 16695.0, E4 = 71.0 / 1920.0, E5 = -17253.0 / 339200.0,
                    E6 = 22.0 / 525.0, E7 = -1.0 / 40.0;

/* Stages 2..6 and the 5th-order solution of one step h from (y, k1)
 * (rk45_adaptive.hpp:210-251).  k[0] must hold k1 on entry. */
static void dp5_solution(double m, double a, const double* y, double h, double k[7][6], double* y5)
{
    double s[6];
    for (int i = 0; i < 6; ++i) s[i] = y[i] + h * (A21 * k[0][i]);
    ks_rhs(s, m, a, k[1]);
    for (int i = 0; i < 6; ++i) s[i] = y[i] + h * (A31 * k[0][i] + A32 * k[1][i]);
    ks_rhs(s, m, a, k[2]);
    for (int i = 0; i < 6; ++i) s[i] = y[i] + h * (A41 * k[0][i] + A42 * k[1][i] + A43 * k[2][i]);
    ks_rhs(s, m, a, k[3]);
    for (int i = 0; i < 6; ++i) s[i] = y[i] + h * (A51 * k[0][i] + A52 * k[1][i] + A53 * k[2][i] + A54 * k[3][i]);
    ks_rhs(s, m, a, k[4]);
    for (int i = 0; i < 6; ++i)
        s[i] = y[i] + h * (A61 * k[0][i] + A62 * k[1][i] + A63 * k[2][i] + A64 * k[3][i] + A65 * k[4][i]);
    ks_rhs(s, m, a, k[5]);
    for (int i = 0; i < 6; ++i)
        y5[i] = y[i] + h * (B1 * k[0][i] + B3 * k[2][i] + B4 * k[3][i] + B5 * k[4][i] + B6 * k[5][i]);
}

/* Mixed absolute/relative max-norm (rk45_adaptive.hpp:254-261), with |h|:
 * the reference multiplies by the signed step, which for h < 0 makes every
 * error non-positive; backward tracing needs the magnitude. */
static double dp45_error(double rtol, double atol, const double* y, const double* yn, double h, double k[7][6])
{
    double e = 0.0;
    for (int i = 0; i < 6; ++i) {
        const double est = fabs(h) * fabs(E1 * k[0][i] + E3 * k[2][i] + E4 * k[3][i] + E5 * k[4][i] + E6 * k[5][i] +
                                        E7 * k[6][i]);
        const double sc = rtol * max_d(fabs(y[i]), fabs(yn[i])) + atol;
        e = max_d(e, est / sc);
    }
    return e;
}

double orc_dp45_attempt(const orc_camera* cam, const double y[6], double h, double y_new[6])
{
    cam_consts c;
    camera_consts(cam, &c);
    double k[7][6];
    ks_rhs(y, c.m, c.a, k[0]);
    dp5_solution(c.m, c.a, y, h, k, y_new);
    ks_rhs(y_new, c.m, c.a, k[6]);
    return dp45_error(cam->rtol, cam->atol, y, y_new, h, k);
}

/* Constraint projection p <- p + alpha n, n = dH/dp, alpha the root of
 * H(p + alpha n) = 0 closest to zero (the closest-root rule of
 * rk45_adaptive.hpp:126-134 applied to the Hamiltonian form). */
static double project_null(double m, double a, double* y, double tol)
{
    const field_t f = ks_field(y, m, a);
    double* p = y + 3;
    const double s = 1.0 + f.k[0] * p[0] + f.k[1] * p[1] + f.k[2] * p[2];
    const double res = 0.5 * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] - 1.0 - 2.0 * f.h * s * s);
    if (!(fabs(res) >= tol)) return fabs(res);
    double n[3];
    for (int i = 0; i < 3; ++i) n[i] = p[i] - 2.0 * f.h * s * f.k[i];
    const double kn = f.k[0] * n[0] + f.k[1] * n[1] + f.k[2] * n[2];
    const double qa = 0.5 * (n[0] * n[0] + n[1] * n[1] + n[2] * n[2] - 2.0 * f.h * kn * kn);
    const double qb = p[0] * n[0] + p[1] * n[1] + p[2] * n[2] - 2.0 * f.h * s * kn;
    const double disc = qb * qb - 4.0 * qa * res;
    if (disc >= 0.0) {
        const double q = -0.5 * (qb + copysign(sqrt(disc), qb));
        if (q != 0.0) {
            const double alpha = res / q;
            for (int i = 0; i < 3; ++i) p[i] += alpha * n[i];
        }
    }
    return fabs(res);
}

static inline double bl_radius(const double* x, double a)
{
    const double a2 = a * a, z2 = x[2] * x[2];
    const double diff = x[0] * x[0] + x[1] * x[1] + z2 - a2;
    return sqrt(max_d(0.5 * (diff + sqrt(diff * diff + 4.0 * a2 * z2)), 1e-24));
}

/* Illinois root of z(theta) on [0, 1] for the 5th-order solution of step
 * theta*h from (y, k1).  Writes the state at the root; returns theta. */
static double disk_root(double m, double a, const double* y, double h, double k1[6], double z0, double z1, double* yr)
{
    double k[7][6];
    memcpy(k[0], k1, sizeof(double) * 6);
    double lo = 0.0, flo = z0, hi = 1.0, fhi = z1;
    int side = 0;
    double t = 1.0;
    double ys[6];
    int have = 0;
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        dp5_solution(m, a, y, t * h, k, ys);
        have = 1;
        const double ft = ys[2];
        if (ft == 0.0 || fabs(hi - lo) < 1e-15 || fabs(ft) < 1e-13 * (1.0 + fabs(ys[0]) + fabs(ys[1]))) break;
        if ((ft > 0.0) == (fhi > 0.0)) {
            hi = t;
            fhi = ft;
            if (side == -1) flo *= 0.5;
            side = -1;
        } else {
            lo = t;
            flo = ft;
            if (side == 1) fhi *= 0.5;
            side = 1;
        }
    }
    if (!have) memcpy(ys, y, sizeof ys);
    memcpy(yr, ys, sizeof ys);
    return t;
}

/* Cubic Hermite interpolant of a step from its end points and FSAL slopes:
 * y(t) = h00 y0 + h10 h f0 + h01 y1 + h11 h f1, t in [0, 1]. */
static void hermite(const double* y0, const double* f0, const double* y1, const double* f1, double h, double t,
                    int n, double* out)
{
    const double t2 = t * t, t3 = t2 * t;
    const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + t;
    const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
    for (int i = 0; i < n; ++i) out[i] = h00 * y0[i] + h10 * h * f0[i] + h01 * y1[i] + h11 * h * f1[i];
}

/* Fraction t of the step where the interpolated r_BL crosses `target`
 * (Illinois on r(x(t)) - target; r(0) and r(1) bracket the target). */
static double crossing_fraction(const double* y0, const double* f0, const double* y1, const double* f1, double h,
                                double a, double target)
{
    double lo = 0.0, hi = 1.0;
    double flo = bl_radius(y0, a) - target, fhi = bl_radius(y1, a) - target;
    if (!((flo > 0.0) != (fhi > 0.0))) return 1.0; /* no bracket: keep the step end */
    int side = 0;
    double t = 1.0, x[3];
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        hermite(y0, f0, y1, f1, h, t, 3, x);
        const double ft = bl_radius(x, a) - target;
        if (ft == 0.0 || fabs(hi - lo) < 1e-15 || fabs(ft) < 1e-13 * target) break;
        if ((ft > 0.0) == (fhi > 0.0)) {
            hi = t;
            fhi = ft;
            if (side == -1) flo *= 0.5;
            side = -1;
        } else {
            lo = t;
            flo = ft;
            if (side == 1) fhi *= 0.5;
            side = 1;
        }
    }
    return t;
}

/* The tracer evaluates the PI30 factor (a step-size heuristic) in FP32 from
 * base-2 logs; the error norm that decides acceptance stays FP64. */
static inline float pi30f(float le, float lp, float order_p1)
{
    return exp2f(-(0.7f / order_p1) * le + (0.3f / order_p1) * (lp - le));
}

/* cont == NULL: the ray ends at its first disk hit (the north-star record).
 * cont != NULL: the translucent-disk continuation of the reference's image
 * path (software_compute_engine.hpp:1734-1765): every crossing on the disk is
 * recorded (radius, azimuth, g) and the ray goes on to its capture or escape,
 * up to ORC_MAX_CROSSINGS crossings; the record `out` still describes the
 * first hit, and cont holds the crossings, the ray's final class and its
 * exit direction. */
/* Boyer-Lindquist (r, theta, phi) of a Kerr-Schild point as Cartesian
 * (spherical_to_cartesian, software_compute_engine.hpp:1063-1066). */
static void bl_cartesian(const double* x, double a, double* out)
{
    double bl[3];
    orc_bl_from_ks(x, a, 0.0, bl);
    const double st = sin(bl[1]);
    out[0] = bl[0] * st * cos(bl[2]);
    out[1] = bl[0] * st * sin(bl[2]);
    out[2] = bl[0] * cos(bl[1]);
}

static void trace_one(const orc_camera* cam, const cam_consts* c, uint32_t px, uint32_t py, orc_ray* out,
                      orc_cont* cont, const orc_fm* fm, double* vol)
{
    const double m = c->m, a = c->a;
    double y[6];
    const double lz0 = initial_state(cam, c, px, py, y);
    const double q0 = orc_carter_q(y, m, a);
    double k[7][6];
    double r = ks_rhs(y, m, a, k[0]);
    double h = -cam->initial_step_fraction * c->r_obs;
    double lambda = 0.0;
    float ln_prev = 0.0f;
    int has_hist = 0;
    double phi_unwrapped;
    {
        double bl[3];
        orc_bl_from_ks(y, a, c->ph_obs, bl);
        phi_unwrapped = bl[2];
    }
    double dH = 0.0;
    uint32_t acc = 0, rej = 0, status = ORC_RAY_UNFINISHED, flags = 0;
    double r_hit = NAN, g = 1.0;
    double yn[6];
    /* continuation: the first hit's record (status, point, lambda, counts, flags, azimuth reference) */
    int hit = 0;
    double y_hit[6], lambda_hit = 0.0, phi_ref_hit = 0.0;
    uint32_t acc_hit = 0, rej_hit = 0, flags_hit = 0;
    if (cont) {
        cont->n_cross = 0;
        cont->fate = ORC_RAY_UNFINISHED;
        cont->exit_dir[0] = cont->exit_dir[1] = cont->exit_dir[2] = NAN;
    }
    /* Certain capture (the CertainAbsorption early-out of
     * carter_ray_classifier.hpp:146-150, used by software_compute_engine.hpp:1356-1368):
     * with no turning point outside r_+ and below the disk's inner edge, an
     * inward ray can only reach the horizon. */
    const double db0 = orc_shadow_distance(m, a, lz0, q0);
    const int can_early = cam->early_capture && db0 > ORC_EARLY_CAPTURE_MARGIN;
    const double r_early = c->disk ? c->r_in : INFINITY;
    const double two_pi = 2.0 * ORC_PI;

    for (uint32_t attempt = 0;; ++attempt) {
        if (r < c->r_capture) {
            status = ORC_RAY_CAPTURED;
            break;
        }
        if (r > c->r_esc) {
            status = ORC_RAY_ESCAPED;
            break;
        }
        if (attempt >= cam->max_steps) {
            flags |= ORC_FLAG_MAX_STEPS;
            break;
        }
        const double cap = cam->step_cap_fraction * max_d(r - c->rh, 0.01 * m);
        if (fabs(h) > cap) h = -cap;
        if (fabs(h) < 1e-8) {
            status = ORC_RAY_CAPTURED;
            flags |= ORC_FLAG_STEP_UNDERFLOW;
            break;
        }
        dp5_solution(m, a, y, h, k, yn);
        const double rn = ks_rhs(yn, m, a, k[6]);
        double err = dp45_error(cam->rtol, cam->atol, y, yn, h, k);
        if (!(err <= 1e300)) err = 1e300; /* non-finite trial: reject with the largest cut */
        if (err <= 1.0) {
            /* accept (rk45_adaptive.hpp:263-302) */
            ++acc;
            int nonfinite = 0;
            for (int i = 0; i < 6; ++i) nonfinite |= !isfinite(yn[i]);
            if (nonfinite) {
                status = ORC_RAY_CAPTURED;
                flags |= ORC_FLAG_NONFINITE;
                break;
            }
            /* disk: first z sign change whose root lies on [r_in, r_out] */
            if (c->disk && y[2] * yn[2] <= 0.0 && y[2] != yn[2]) {
                const double sl = y[2] / (y[2] - yn[2]);
                const double xe = y[0] + sl * (yn[0] - y[0]);
                const double ye = y[1] + sl * (yn[1] - y[1]);
                const double re = sqrt(max_d(xe * xe + ye * ye - a * a, 0.0));
                const double margin = 0.05 * re + 0.5 * m;
                if (re >= c->r_in - margin && re <= c->r_out + margin) {
                    double yr[6];
                    const double t = disk_root(m, a, y, h, k[0], y[2], yn[2], yr);
                    const double rr = bl_radius(yr, a);
                    if (rr >= c->r_in && rr <= c->r_out && rr > c->rh * 1.02) {
                        if (!cont) {
                            status = ORC_RAY_DISK;
                            r_hit = rr;
                            g = orc_redshift_at(m, a, rr, lz0);
                            lambda += t * h;
                            memcpy(y, yr, sizeof yr);
                            break;
                        }
                        /* record the crossing and go on through the disk */
                        double bl[3];
                        orc_bl_from_ks(yr, a, phi_unwrapped, bl);
                        const uint32_t kx = cont->n_cross++;
                        cont->cross_r[kx] = rr;
                        cont->cross_phi[kx] = bl[2];
                        cont->cross_g[kx] = orc_redshift_at(m, a, rr, lz0);
                        if (!hit) {
                            hit = 1;
                            r_hit = rr;
                            g = cont->cross_g[kx];
                            memcpy(y_hit, yr, sizeof yr);
                            lambda_hit = lambda + t * h;
                            phi_ref_hit = phi_unwrapped;
                            acc_hit = acc;
                            rej_hit = rej;
                            flags_hit = flags;
                        }
                        if (cont->n_cross >= ORC_MAX_CROSSINGS) break;
                    }
                }
            }
            /* capture / escape / certain capture inside this step: the terminal
             * point is interpolated to the threshold radius, so it does not
             * depend on where the step happened to end */
            {
                double target = 0.0;
                uint32_t term = 0, tflag = 0;
                if (rn < c->r_capture) {
                    term = ORC_RAY_CAPTURED;
                    target = c->r_capture;
                } else if (rn > c->r_esc) {
                    term = ORC_RAY_ESCAPED;
                    target = c->r_esc;
                } else if (can_early && rn < r_early) {
                    /* dr_BL/dlambda from dx/dlambda (kerr_invariants.hpp:140); the trace
                     * runs towards decreasing lambda, so dr/dlambda > 0 means inwards. */
                    const double r2 = rn * rn, z = yn[2];
                    const double drdl = (r2 * rn * (yn[0] * k[6][0] + yn[1] * k[6][1]) +
                                         rn * (r2 + a * a) * z * k[6][2]) /
                                        (r2 * r2 + a * a * z * z);
                    if (drdl > 0.0) {
                        term = ORC_RAY_CAPTURED;
                        tflag = ORC_FLAG_EARLY_CAPTURE;
                        target = r_early;
                    }
                }
                if (term) {
                    const double t = crossing_fraction(y, k[0], yn, k[6], h, a, target);
                    double yt[6];
                    hermite(y, k[0], yn, k[6], h, t, 6, yt);
                    memcpy(y, yt, sizeof yt);
                    lambda += t * h;
                    status = term;
                    flags |= tflag;
                    break;
                }
            }
            dH = max_d(dH, project_null(m, a, yn, cam->projection_tol));
            if (fm) { /* hydro model 2: the step's chord through the torus (:1725-1731) */
                double from[3], to[3];
                bl_cartesian(y, a, from);
                bl_cartesian(yn, a, to);
                orc_fm_accumulate(fm, from, to, lz0, vol);
            }
            /* phi unwrapping, kerr_schild_null_integrator.hpp:61-63 */
            {
                const double raw = atan2(yn[1], yn[0]) - atan2(a, rn);
                double d = raw - phi_unwrapped;
                d -= two_pi * floor(d / two_pi + 0.5);
                phi_unwrapped += d;
            }
            lambda += h;
            memcpy(y, yn, sizeof yn);
            memcpy(k[0], k[6], sizeof(double) * 6); /* FSAL */
            r = rn;
            float factor = 5.0f;
            if (err != 0.0) {
                const float le = log2f(fmaxf((float)err, 1e-12f));
                factor = pi30f(le, has_hist ? ln_prev : le, 5.0f);
                ln_prev = le;
                has_hist = 1;
            }
            double ah = fabs(h) * clamp_d(0.9 * factor, 0.2, 5.0);
            ah = clamp_d(ah, 1e-8, 1e13);
            h = -ah;
        } else {
            /* reject (rk45_adaptive.hpp:303-311) */
            ++rej;
            const float le = log2f(fmaxf((float)err, 1e-12f));
            const float factor = pi30f(le, has_hist ? ln_prev : le, 4.0f);
            ln_prev = le;
            has_hist = 1;
            h = -fabs(h) * clamp_d(0.9 * factor, 0.1, 0.9);
        }
    }

    if (cont) {
        cont->fate = status;
        {  /* the sky-lookup direction at the ray's end */
            double dy[6];
            ks_rhs(y, m, a, dy);
            const double len = sqrt(dy[0] * dy[0] + dy[1] * dy[1] + dy[2] * dy[2]);
            const double inv = 1.0 / max_d(len, 1e-12);
            for (int i = 0; i < 3; ++i) cont->exit_dir[i] = -dy[i] * inv;
        }
        if (hit) {
            /* the record describes the first hit */
            status = ORC_RAY_DISK;
            memcpy(y, y_hit, sizeof y_hit);
            lambda = lambda_hit;
            phi_unwrapped = phi_ref_hit;
            acc = acc_hit;
            rej = rej_hit;
            flags = flags_hit;
        }
    }
    double bl[3];
    orc_bl_from_ks(y, a, phi_unwrapped, bl);
    out->status = status;
    out->flags = flags;
    out->steps_accepted = acc;
    out->steps_rejected = rej;
    out->r = bl[0];
    out->theta = bl[1];
    out->phi = bl[2];
    out->r_hit = r_hit;
    out->g = g;
    out->lambda = lambda;
    out->dH = dH;
    out->dE = energy_from_null(y, m, a) - 1.0;
    out->dLz = (y[0] * y[4] - y[1] * y[3]) - lz0;
    out->dQ = orc_carter_q(y, m, a) - q0;
    out->db_shadow = db0;
    out->body = (status == ORC_RAY_DISK || status == ORC_RAY_CAPTURED) ? 0u : ORC_BODY_NONE;
    /* sky-lookup direction of an escaped ray: minus the normalised dx/dlambda of
     * the terminal state (software_compute_engine.hpp:1771-1775) */
    out->exit_dir[0] = out->exit_dir[1] = out->exit_dir[2] = NAN;
    if (status == ORC_RAY_ESCAPED) {
        double dy[6];
        ks_rhs(y, m, a, dy);
        const double len = sqrt(dy[0] * dy[0] + dy[1] * dy[1] + dy[2] * dy[2]);
        const double inv = 1.0 / max_d(len, 1e-12);
        for (int i = 0; i < 3; ++i) out->exit_dir[i] = -dy[i] * inv;
    }
}

typedef struct {
    const orc_camera* cam;
    const cam_consts* c;
    const uint64_t* idx;
    uint64_t first, count;
    orc_ray* out;
    orc_cont* cont;
    const orc_fm* fm;
    double* vol;
    atomic_ullong next;
} work_t;

static void* worker(void* arg)
{
    work_t* w = (work_t*)arg;
    const uint64_t chunk = 16;
    for (;;) {
        const uint64_t b = atomic_fetch_add(&w->next, chunk);
        if (b >= w->count) break;
        const uint64_t e = (b + chunk < w->count) ? b + chunk : w->count;
        for (uint64_t i = b; i < e; ++i) {
            const uint64_t pix = w->idx ? w->idx[i] : w->first + i;
            const uint32_t px = (uint32_t)(pix % w->cam->screen_width);
            const uint32_t py = (uint32_t)(pix / w->cam->screen_width);
            trace_one(w->cam, w->c, px, py, &w->out[i], w->cont ? &w->cont[i] : NULL, w->fm,
                      w->vol ? w->vol + 6 * i : NULL);
        }
    }
    return NULL;
}

static void trace_range(const orc_camera* cam, const uint64_t* pixel_index, uint64_t first, uint64_t count,
                        orc_ray* out, orc_cont* cont, const orc_fm* fm, double* vol, int threads);

void orc_trace(const orc_camera* cam, const uint64_t* pixel_index, uint64_t first, uint64_t count, orc_ray* out,
               int threads)
{
    trace_range(cam, pixel_index, first, count, out, NULL, NULL, NULL, threads);
}

void orc_trace_cont(const orc_camera* cam, const uint64_t* pixel_index, uint64_t first, uint64_t count,
                    orc_ray* out, orc_cont* cont, int threads)
{
    trace_range(cam, pixel_index, first, count, out, cont, NULL, NULL, threads);
}

void orc_trace_volume(const orc_camera* cam, const orc_fm* fm, const uint64_t* pixel_index, uint64_t first,
                      uint64_t count, orc_ray* out, orc_cont* cont, double* vol, int threads)
{
    memset(vol, 0, sizeof(double) * 6 * count);
    trace_range(cam, pixel_index, first, count, out, cont, fm, vol, threads);
}

static void trace_range(const orc_camera* cam, const uint64_t* pixel_index, uint64_t first, uint64_t count,
                        orc_ray* out, orc_cont* cont, const orc_fm* fm, double* vol, int threads)
{
    cam_consts c;
    camera_consts(cam, &c);
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    work_t w;
    w.cam = cam;
    w.c = &c;
    w.idx = pixel_index;
    w.first = first;
    w.count = count;
    w.out = out;
    w.cont = cont;
    w.fm = fm;
    w.vol = vol;
    atomic_init(&w.next, 0);
    if (threads == 1) {
        worker(&w);
        return;
    }
    pthread_t* tid = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    int started = 0;
    for (int t = 0; t < threads; ++t)
        if (pthread_create(&tid[t], NULL, worker, &w) == 0) ++started;
    if (started == 0) worker(&w);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    free(tid);
}
