/*
 * bl_oracle.c -- FP64 CPU oracle of the Boyer-Lindquist Kerr-Newman tracer.
 *
 * TEST INFRASTRUCTURE ONLY (same rules as ks_oracle.c): a plain-C restatement
 * used as the checker of the CUDA Boyer-Lindquist kernel.
 *
 * What it restates (reference = Wartets/Relativity-Simulator):
 *   - Kerr-Newman metric in Boyer-Lindquist coordinates (G = c = k_e = 1)
 *       include/relativistic/metrics/kerr_newman.hpp:141-169; outer horizon :95-101
 *     (KerrMetric, metrics/kerr.hpp:119-146, is the Q = 0 case)
 *   - its r- and theta-derivatives  kerr_newman.hpp:203-251
 *   - geodesic acceleration -Gamma^mu_ab u^a u^b
 *       include/relativistic/integrators/rk45_adaptive.hpp:64-88
 *     contracted in factored form (bl_rhs below) instead of forming Gamma
 *   - ZAMO tetrad  include/relativistic/observer/observer_tetrad.hpp:82-100 and the
 *     light ray u = e0 + sum_i n_i e_i  :144-166 with n = -(n_r, n_th, n_ph)
 *       software_compute_engine.hpp:1347-1350
 *   - radii of metric type 5  software_compute_engine.hpp:3364-3368 (r_+ of the
 *     Kerr-Newman metric, ISCO from the Kerr formula of :1052-1061)
 *   - projection onto the null cone by solving for u^t, closest root
 *       rk45_adaptive.hpp:91-139
 *   - pole reflection  software_compute_engine.hpp:1492-1500
 *   - disk: crossing of theta = pi/2 with r on [r_in, r_out] and r > 1.02 r_+
 *       :1538-1547, g = redshift_at(m, a, r, L/E)  :1551-1556
 *   - Carter constant  include/relativistic/metrics/kerr_invariants.hpp:21-58 (mu = 0)
 * The reference steps this path with heuristic RK4 (software_compute_engine.hpp:
 * 1434-1479); like the Kerr-Schild oracle, this one runs the DP45 + PI30 +
 * step-cap machinery of RK45AdaptiveIntegrator on the state
 * y = (r, theta, phi, u^t, u^r, u^theta, u^phi) with steps h < 0 (t enters no
 * right-hand side and is not integrated).  The Carter certain-capture test of
 * the Kerr path (software_compute_engine.hpp:1356-1368) is applied with the
 * Kerr-Newman radial potential (Delta includes Q^2).
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "ks_oracle.h"

#define ORC_PI 3.14159265358979323846
#define HALF_PI (0.5 * ORC_PI)

static inline double max_d(double a, double b) { return (a < b) ? b : a; }
static inline double clamp_d(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

double orc_kn_horizon(double mass, double spin, double charge)
{
    const double diff = mass * mass - spin * spin - charge * charge;
    return (diff < 0.0) ? mass : mass + sqrt(diff);
}

/* Metric components g = (g_tt, g_tphi, g_rr, g_thth, g_phiphi) and their r- and
 * theta-derivatives.  With F = (2 M r - Q^2) / rho^2:
 *   g_tt = F - 1, g_tphi = -a s^2 F, g_rr = rho^2 / Delta, g_thth = rho^2,
 *   g_phiphi = s^2 (r^2 + a^2 + a^2 s^2 F)   (= Sigma s^2 / rho^2). */
typedef struct {
    double g[5], dr[5], dth[5];
    double delta, rho2, sin2;
} kn_geom;

static void kn_geometry(double m, double a, double q2, double r, double th, kn_geom* G)
{
    const double s = sin(th), c = cos(th);
    const double s2 = s * s, c2 = c * c, sc = s * c;
    const double a2 = a * a, r2 = r * r;
    const double rho2 = r2 + a2 * c2;
    const double irho2 = 1.0 / rho2;
    const double delta = r2 - 2.0 * m * r + a2 + q2;
    const double idelta = 1.0 / delta;
    const double F = (2.0 * m * r - q2) * irho2;
    const double dFr = (2.0 * m - 2.0 * r * F) * irho2;
    const double dFt = 2.0 * a2 * sc * F * irho2;
    const double W = r2 + a2 + a2 * s2 * F;
    G->g[0] = F - 1.0;
    G->g[1] = -a * s2 * F;
    G->g[2] = rho2 * idelta;
    G->g[3] = rho2;
    G->g[4] = s2 * W;
    G->dr[0] = dFr;
    G->dr[1] = -a * s2 * dFr;
    G->dr[2] = (2.0 * r - G->g[2] * (2.0 * r - 2.0 * m)) * idelta;
    G->dr[3] = 2.0 * r;
    G->dr[4] = s2 * (2.0 * r + a2 * s2 * dFr);
    G->dth[0] = dFt;
    G->dth[1] = -a * (2.0 * sc * F + s2 * dFt);
    G->dth[2] = -2.0 * a2 * sc * idelta;
    G->dth[3] = -2.0 * a2 * sc;
    G->dth[4] = 2.0 * sc * W + s2 * a2 * (2.0 * sc * F + s2 * dFt);
    G->delta = delta;
    G->rho2 = rho2;
    G->sin2 = s2;
}

void orc_kn_metric(double mass, double spin, double charge, double r, double theta, double g[5])
{
    kn_geom G;
    kn_geometry(mass, spin, charge * charge, r, theta, &G);
    memcpy(g, G.g, sizeof G.g);
}

void orc_kn_metric_derivs(double mass, double spin, double charge, double r, double theta, double dr[5],
                          double dth[5])
{
    kn_geom G;
    kn_geometry(mass, spin, charge * charge, r, theta, &G);
    memcpy(dr, G.dr, sizeof G.dr);
    memcpy(dth, G.dth, sizeof G.dth);
}

/* du^mu/dlambda = -Gamma^mu_ab u^a u^b from the Euler-Lagrange form of the
 * geodesic equation, d(g_mu nu u^nu)/dlambda = (1/2) d_mu g_ab u^a u^b:
 *   r, theta:  g_rr a^r = (1/2) d_r g(u,u) - (d_r g_rr u^r + d_th g_rr u^th) u^r  (same for theta)
 *   t, phi:    [g_tt g_tphi; g_tphi g_phiphi] (a^t, a^phi) = -(dg/dlambda) (u^t, u^phi),
 *              whose determinant is -Delta sin^2 theta. */
static void bl_rhs(double m, double a, double q2, const double* y, double* dy)
{
    kn_geom G;
    kn_geometry(m, a, q2, y[0], y[1], &G);
    const double ut = y[3], ur = y[4], uth = y[5], up = y[6];
    const double half_r = 0.5 * (G.dr[0] * ut * ut + 2.0 * G.dr[1] * ut * up + G.dr[2] * ur * ur + G.dr[3] * uth * uth +
                                 G.dr[4] * up * up);
    const double half_t = 0.5 * (G.dth[0] * ut * ut + 2.0 * G.dth[1] * ut * up + G.dth[2] * ur * ur +
                                 G.dth[3] * uth * uth + G.dth[4] * up * up);
    const double ar = (half_r - (G.dr[2] * ur + G.dth[2] * uth) * ur) * (G.delta / G.rho2);
    const double ath = (half_t - (G.dr[3] * ur + G.dth[3] * uth) * uth) / G.rho2;
    const double dgtt = G.dr[0] * ur + G.dth[0] * uth;
    const double dgtp = G.dr[1] * ur + G.dth[1] * uth;
    const double dgpp = G.dr[4] * ur + G.dth[4] * uth;
    const double bt = -(dgtt * ut + dgtp * up);
    const double bp = -(dgtp * ut + dgpp * up);
    const double idet = -1.0 / (G.delta * max_d(G.sin2, 1e-30));
    dy[0] = ur;
    dy[1] = uth;
    dy[2] = up;
    dy[3] = (G.g[4] * bt - G.g[1] * bp) * idet;
    dy[4] = ar;
    dy[5] = ath;
    dy[6] = (G.g[0] * bp - G.g[1] * bt) * idet;
}

void orc_bl_rhs(double mass, double spin, double charge, const double y[7], double dy[7])
{
    bl_rhs(mass, spin, charge * charge, y, dy);
}

/* (1/2) g(u, u) */
static double null_residual(double m, double a, double q2, const double* y)
{
    kn_geom G;
    kn_geometry(m, a, q2, y[0], y[1], &G);
    const double ut = y[3], ur = y[4], uth = y[5], up = y[6];
    return 0.5 * (G.g[0] * ut * ut + 2.0 * G.g[1] * ut * up + G.g[2] * ur * ur + G.g[3] * uth * uth +
                  G.g[4] * up * up);
}

double orc_bl_null_residual(double mass, double spin, double charge, const double y[7])
{
    return null_residual(mass, spin, charge * charge, y);
}

/* E = -u_t, L = u_phi, Carter Q = u_theta^2 + cos^2(theta) (L^2 / sin^2 - a^2 E^2). */
static void invariants(double m, double a, double q2, const double* y, double out[3])
{
    kn_geom G;
    kn_geometry(m, a, q2, y[0], y[1], &G);
    const double E = -(G.g[0] * y[3] + G.g[1] * y[6]);
    const double L = G.g[1] * y[3] + G.g[4] * y[6];
    const double pth = G.g[3] * y[5];
    const double c = cos(y[1]);
    out[0] = E;
    out[1] = L;
    out[2] = pth * pth + c * c * (L * L / max_d(G.sin2, 1e-30) - a * a * E * E);
}

void orc_bl_invariants(double mass, double spin, double charge, const double y[7], double out[3])
{
    invariants(mass, spin, charge * charge, y, out);
}

/* Signed distance (in impact parameter, units of M) of (xi, eta) from the
 * Kerr-Newman critical curve: the smallest local minimum of the radial
 * potential R(r) = (r^2 + a^2 - a xi)^2 - Delta (eta + (xi - a)^2) outside r_+
 * (carter_ray_classifier.hpp:132-135 with Delta = r^2 - 2 M r + a^2 + Q^2)
 * moved to zero by d_eta = R_min / Delta.  > 0: no turning point. */
double orc_kn_shadow_distance(double mass, double spin, double charge, double xi, double eta)
{
    const double a = spin, a2 = a * a, q2 = charge * charge;
    const double rp = orc_kn_horizon(mass, spin, charge);
    const double K = eta + (xi - a) * (xi - a);
    const double P = a2 - xi * xi - eta;
    const double Qc = 2.0 * mass * K;
    const double R0 = -a2 * eta - q2 * K;
    /* stationary points: 4 r^3 + 2 P r + Qc = 0 */
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
    double best = INFINITY, best_r = 0.0;
    for (int i = 0; i < n; ++i) {
        const double r = roots[i];
        if (!(r > rp)) continue;
        if (12.0 * r * r + 2.0 * P <= 0.0) continue;
        const double R = ((r * r + P) * r + Qc) * r + R0;
        if (R < best) {
            best = R;
            best_r = r;
        }
    }
    if (!isfinite(best)) return INFINITY;
    const double delta = best_r * best_r - 2.0 * mass * best_r + a2 + q2;
    const double b = sqrt(max_d(eta + xi * xi, 1e-30));
    return best / max_d(delta, 1e-30) / (2.0 * b);
}

/* ZAMO light ray at (r, theta): u = e0 - (n_r e_r + n_th e_th + n_ph e_ph) with
 * e0 = (1, 0, 0, omega) / alpha, omega = -g_tphi / g_phiphi,
 * alpha^2 = -(g_tt + omega g_tphi), e_i the unit coordinate vectors (already
 * orthogonal to e0 and to each other, so the Gram-Schmidt pass of
 * observer_tetrad.hpp:104-141 changes them only by rounding). */
static void zamo_ray(double m, double a, double q2, double r, double th, double n_r, double n_th, double n_ph,
                     double u[4])
{
    kn_geom G;
    kn_geometry(m, a, q2, r, th, &G);
    const double omega = -G.g[1] / G.g[4];
    const double alpha = sqrt(max_d(-(G.g[0] + omega * G.g[1]), 1e-30));
    const double len = sqrt(n_r * n_r + n_th * n_th + n_ph * n_ph);
    const double inv = (len > 0.0) ? 1.0 / len : 1.0;
    u[0] = 1.0 / alpha;
    u[1] = -n_r * inv / sqrt(max_d(G.g[2], 1e-30));
    u[2] = -n_th * inv / sqrt(max_d(G.g[3], 1e-30));
    u[3] = omega / alpha - n_ph * inv / sqrt(max_d(G.g[4], 1e-30));
}

void orc_bl_zamo_ray(double mass, double spin, double charge, double r, double theta, double n_r, double n_th,
                     double n_ph, double u[4])
{
    zamo_ray(mass, spin, charge * charge, r, theta, n_r, n_th, n_ph, u);
}

/* ---------------------------------------------------------------------- */
typedef struct {
    double m, a, q2, rh;
    double r_obs, th_obs, ph_obs;
    double aspect, fov;
    double fwd[3], rgt[3], up[3];
    double r_in, r_out, r_capture, r_esc;
    int disk;
} bl_consts;

static void bl_camera_consts(const orc_camera* cam, double charge, bl_consts* c)
{
    c->m = max_d(cam->metric_mass, 1e-4);
    c->a = clamp_d(cam->metric_spin, -0.999 * c->m, 0.999 * c->m);
    c->q2 = charge * charge;
    c->rh = orc_kn_horizon(c->m, c->a, charge);
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

/* software_compute_engine.hpp:3843-3862 (pixel -> world direction), :3912-3938
 * (spherical components at the observer), :1347-1350 (ZAMO ray). */
static void bl_initial_state(const orc_camera* cam, const bl_consts* c, uint32_t px, uint32_t py, double y0[7])
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
    const double n_ph = d[0] * (-sp) + d[1] * cp;
    y0[0] = c->r_obs;
    y0[1] = c->th_obs;
    y0[2] = c->ph_obs;
    zamo_ray(c->m, c->a, c->q2, c->r_obs, c->th_obs, n_r, n_th, n_ph, y0 + 3);
}

void orc_bl_initial_state(const orc_camera* cam, double charge, uint32_t px, uint32_t py, double y0[7])
{
    bl_consts c;
    bl_camera_consts(cam, charge, &c);
    bl_initial_state(cam, &c, px, py, y0);
}

/* Dormand-Prince 5(4) (rk45_adaptive.hpp:196-203) and its continuous extension
 * of order 4 (Hairer, Norsett & Wanner, Solving ODEs I, sec. II.6). */
static const double A21 = 1.0 / 5.0;
static const double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
static const double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
static const double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0, A54 = -212.0 / 729.0;
static const double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0, A64 = 49.0 / 176.0,
                    A65 = -5103.0 / 18656.0;
static const double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0, B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
static const double E1 = 71.0 / 57600.0, E3 = -71.0 / 16695.0, E4 = 71.0 / 1920.0, E5 = -17253.0 / 339200.0,
                    E6 = 22.0 / 525.0, E7 = -1.0 / 40.0;
static const double D1 = -12715105075.0 / 11282082432.0, D3 = 87487479700.0 / 32700410799.0,
                    D4 = -10690763975.0 / 1880347072.0, D5 = 701980252875.0 / 199316789632.0,
                    D6 = -1453857185.0 / 822651844.0, D7 = 69997945.0 / 29380423.0;

#define NB 7

static void stages(const bl_consts* c, const double* y, double h, double k[7][NB], double* y5)
{
    double s[NB];
    for (int i = 0; i < NB; ++i) s[i] = y[i] + h * (A21 * k[0][i]);
    bl_rhs(c->m, c->a, c->q2, s, k[1]);
    for (int i = 0; i < NB; ++i) s[i] = y[i] + h * (A31 * k[0][i] + A32 * k[1][i]);
    bl_rhs(c->m, c->a, c->q2, s, k[2]);
    for (int i = 0; i < NB; ++i) s[i] = y[i] + h * (A41 * k[0][i] + A42 * k[1][i] + A43 * k[2][i]);
    bl_rhs(c->m, c->a, c->q2, s, k[3]);
    for (int i = 0; i < NB; ++i) s[i] = y[i] + h * (A51 * k[0][i] + A52 * k[1][i] + A53 * k[2][i] + A54 * k[3][i]);
    bl_rhs(c->m, c->a, c->q2, s, k[4]);
    for (int i = 0; i < NB; ++i)
        s[i] = y[i] + h * (A61 * k[0][i] + A62 * k[1][i] + A63 * k[2][i] + A64 * k[3][i] + A65 * k[4][i]);
    bl_rhs(c->m, c->a, c->q2, s, k[5]);
    for (int i = 0; i < NB; ++i)
        y5[i] = y[i] + h * (B1 * k[0][i] + B3 * k[2][i] + B4 * k[3][i] + B5 * k[4][i] + B6 * k[5][i]);
}

/* Max-norm error with |h| (rk45_adaptive.hpp:254-261 multiplies by the signed step). */
static double dp45_error(double rtol, double atol, const double* y, const double* yn, double h, double k[7][NB])
{
    double e = 0.0;
    for (int i = 0; i < NB; ++i) {
        const double est = fabs(h) * fabs(E1 * k[0][i] + E3 * k[2][i] + E4 * k[3][i] + E5 * k[4][i] + E6 * k[5][i] +
                                        E7 * k[6][i]);
        const double sc = rtol * max_d(fabs(y[i]), fabs(yn[i])) + atol;
        e = max_d(e, est / sc);
    }
    return e;
}

static void dense(const double* y0, const double* y1, double k[7][NB], double h, double t, double* out)
{
    for (int i = 0; i < NB; ++i) {
        const double d = y1[i] - y0[i];
        const double b = h * k[0][i] - d;
        const double cc = d - h * k[6][i] - b;
        const double e = h * (D1 * k[0][i] + D3 * k[2][i] + D4 * k[3][i] + D5 * k[4][i] + D6 * k[5][i] + D7 * k[6][i]);
        out[i] = y0[i] + t * (d + (1.0 - t) * (b + t * (cc + (1.0 - t) * e)));
    }
}

/* Illinois root on [0, 1] of theta(t) - pi/2 on the dense output. */
static double equator_root(const double* y0, const double* y1, double k[7][NB], double h, double f0, double f1)
{
    double lo = 0.0, hi = 1.0, flo = f0, fhi = f1, t = 1.0, yy[NB];
    int side = 0;
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        dense(y0, y1, k, h, t, yy);
        const double ft = yy[1] - HALF_PI;
        if (ft == 0.0 || fabs(hi - lo) < 1e-15 || fabs(ft) < 1e-15) break;
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

/* Fraction of the step where r of the dense output crosses target (Illinois). */
static double radius_crossing(const double* y0, const double* y1, double k[7][NB], double h, double target)
{
    double lo = 0.0, hi = 1.0, x[NB];
    double flo = y0[0] - target, fhi = y1[0] - target;
    if (!((flo > 0.0) != (fhi > 0.0))) return 1.0;
    int side = 0;
    double t = 1.0;
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        dense(y0, y1, k, h, t, x);
        const double ft = x[0] - target;
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

/* u^t <- the root of g(u, u) = 0 closest to the current u^t
 * (rk45_adaptive.hpp:91-139), from the cancellation-free pair q / A, C / q.
 * Returns |(1/2) g(u, u)| before. */
static double project_null(const bl_consts* c, double* y, double tol)
{
    kn_geom G;
    kn_geometry(c->m, c->a, c->q2, y[0], y[1], &G);
    const double ut = y[3], ur = y[4], uth = y[5], up = y[6];
    const double A = G.g[0];
    const double B = 2.0 * G.g[1] * up;
    const double C = G.g[2] * ur * ur + G.g[3] * uth * uth + G.g[4] * up * up;
    const double res = 0.5 * ((A * ut + B) * ut + C);
    if (!(fabs(res) >= tol)) return fabs(res);
    const double disc = B * B - 4.0 * A * C;
    if (disc >= 0.0) {
        const double q = -0.5 * (B + copysign(sqrt(disc), B));
        double best = ut, dist = INFINITY;
        if (A != 0.0) {
            const double x = q / A;
            if (fabs(x - ut) < dist) {
                dist = fabs(x - ut);
                best = x;
            }
        }
        if (q != 0.0) {
            const double x = C / q;
            if (fabs(x - ut) < dist) {
                dist = fabs(x - ut);
                best = x;
            }
        }
        y[3] = best;
    }
    return fabs(res);
}

/* theta outside [0, pi]: the same point with theta reflected and phi + pi
 * (software_compute_engine.hpp:1492-1500).  f (a state derivative) follows. */
static void reflect_pole(double* y, double* f)
{
    if (y[1] < 0.0) {
        y[1] = -y[1];
    } else if (y[1] > ORC_PI) {
        y[1] = 2.0 * ORC_PI - y[1];
    } else {
        return;
    }
    y[2] += ORC_PI;
    y[5] = -y[5];
    if (f) {
        f[1] = -f[1];
        f[5] = -f[5];
    }
}

static inline float pi30f(float le, float lp, float order_p1)
{
    return exp2f(-(0.7f / order_p1) * le + (0.3f / order_p1) * (lp - le));
}

/* cont != NULL: the translucent-disk continuation (as orc_trace_cont in
 * ks_oracle.c; software_compute_engine.hpp:1538-1560 for this path): every
 * crossing on the disk is recorded at the reflected root point and the ray
 * goes on; `out` still describes the first hit. */
/* Sky-lookup direction of a (pole-reflected) state: the orthonormal-frame
 * velocity mapped to a Cartesian direction of travel (software_compute_engine.hpp:
 * 1581-1589 with local_frame_to_travel_direction, :1148-1168). */
static void exit_direction(double m, double a, double q2, const double* y, double* e)
{
    kn_geom G;
    kn_geometry(m, a, q2, y[0], y[1], &G);
    const double* gm = G.g;
    const double st = sin(y[1]), ct = cos(y[1]), sp = sin(y[2]), cp = cos(y[2]);
    const double lr = sqrt(fmax(gm[2], 0.0)) * y[4], lt = sqrt(fmax(gm[3], 0.0)) * y[5], lp = sqrt(fmax(gm[4], 0.0)) * y[6];
    const double x = -(lr * st * cp + lt * ct * cp - lp * sp);
    const double yy = -(lr * st * sp + lt * ct * sp + lp * cp);
    const double z = -(lr * ct - lt * st);
    const double len = sqrt(x * x + yy * yy + z * z);
    if (len <= 1e-12) {
        e[0] = 1.0;
        e[1] = e[2] = 0.0;
    } else {
        e[0] = x / len;
        e[1] = yy / len;
        e[2] = z / len;
    }
}

/* spherical_to_cartesian (software_compute_engine.hpp:1063-1066) */
static void sph_cartesian(const double* y, double* out)
{
    const double st = sin(y[1]);
    out[0] = y[0] * st * cos(y[2]);
    out[1] = y[0] * st * sin(y[2]);
    out[2] = y[0] * cos(y[1]);
}

static void trace_one(const orc_camera* cam, const bl_consts* c, uint32_t px, uint32_t py, orc_ray* out,
                      orc_cont* cont, const orc_fm* fm, double* vol)
{
    const double m = c->m, a = c->a, q2 = c->q2;
    double y[NB];
    bl_initial_state(cam, c, px, py, y);
    double inv0[3];
    invariants(m, a, q2, y, inv0);
    const double E0 = inv0[0];
    double k[7][NB];
    bl_rhs(m, a, q2, y, k[0]);
    double h = -cam->initial_step_fraction * c->r_obs;
    double lambda = 0.0, dH = 0.0;
    float ln_prev = 0.0f;
    int has_hist = 0;
    uint32_t acc = 0, rej = 0, status = ORC_RAY_UNFINISHED, flags = 0;
    double r_hit = NAN, g = 1.0;
    double yn[NB];
    const double xi = inv0[1] / E0, eta = inv0[2] / (E0 * E0);
    const double db0 = orc_kn_shadow_distance(m, a, sqrt(q2), xi, eta);
    const int can_early = cam->early_capture && db0 > ORC_EARLY_CAPTURE_MARGIN;
    const double r_early = c->disk ? c->r_in : INFINITY;
    int hit = 0;
    double y_hit[NB], lambda_hit = 0.0;
    uint32_t acc_hit = 0, rej_hit = 0, flags_hit = 0;
    if (cont) {
        cont->n_cross = 0;
        cont->fate = ORC_RAY_UNFINISHED;
        cont->exit_dir[0] = cont->exit_dir[1] = cont->exit_dir[2] = NAN;
    }

    for (uint32_t attempt = 0;; ++attempt) {
        const double r = y[0];
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
        stages(c, y, h, k, yn);
        bl_rhs(m, a, q2, yn, k[6]);
        double err = dp45_error(cam->rtol, cam->atol, y, yn, h, k);
        if (!(err <= 1e300)) err = 1e300;
        if (err > 1.0) {
            ++rej;
            const float le = log2f(fmaxf((float)err, 1e-12f));
            const float factor = pi30f(le, has_hist ? ln_prev : le, 4.0f);
            ln_prev = le;
            has_hist = 1;
            h = -fabs(h) * clamp_d(0.9 * factor, 0.1, 0.9);
            continue;
        }
        ++acc;
        int nonfinite = 0;
        for (int i = 0; i < NB; ++i) nonfinite |= !isfinite(yn[i]);
        if (nonfinite) {
            status = ORC_RAY_CAPTURED;
            flags |= ORC_FLAG_NONFINITE;
            break;
        }
        /* disk: theta = pi/2 crossing whose root lies on [r_in, r_out] */
        {
            const double f0 = y[1] - HALF_PI, f1 = yn[1] - HALF_PI;
            if (c->disk && f0 * f1 <= 0.0 && f0 != f1) {
                const double sl = f0 / (f0 - f1);
                const double re = y[0] + sl * (yn[0] - y[0]);
                const double margin = 0.05 * re + 0.5 * m;
                if (re >= c->r_in - margin && re <= c->r_out + margin) {
                    const double t = equator_root(y, yn, k, h, f0, f1);
                    double yr[NB];
                    dense(y, yn, k, h, t, yr);
                    const double rr = yr[0];
                    if (rr >= c->r_in && rr <= c->r_out && rr > c->rh * 1.02) {
                        double iv[3];
                        invariants(m, a, q2, yr, iv);
                        const double gg = orc_redshift_at(m, a, rr, iv[1] / iv[0]);
                        if (!cont) {
                            status = ORC_RAY_DISK;
                            r_hit = rr;
                            g = gg;
                            lambda += t * h;
                            memcpy(y, yr, sizeof yr);
                            break;
                        }
                        double yp[NB];
                        memcpy(yp, yr, sizeof yr);
                        reflect_pole(yp, NULL);
                        const uint32_t kx = cont->n_cross++;
                        cont->cross_r[kx] = rr;
                        cont->cross_phi[kx] = yp[2];
                        cont->cross_g[kx] = gg;
                        if (!hit) {
                            hit = 1;
                            r_hit = rr;
                            g = gg;
                            memcpy(y_hit, yr, sizeof yr);
                            lambda_hit = lambda + t * h;
                            acc_hit = acc;
                            rej_hit = rej;
                            flags_hit = flags;
                        }
                        if (cont->n_cross >= ORC_MAX_CROSSINGS) break;
                    }
                }
            }
        }
        /* capture / escape / certain capture inside this step, the terminal point on the
         * dense output at the threshold radius */
        {
            double target = 0.0;
            uint32_t term = 0, tflag = 0;
            const double rn = yn[0];
            if (rn < c->r_capture) {
                term = ORC_RAY_CAPTURED;
                target = c->r_capture;
            } else if (rn > c->r_esc) {
                term = ORC_RAY_ESCAPED;
                target = c->r_esc;
            } else if (can_early && rn < r_early && yn[4] > 0.0) {
                /* u^r > 0 with h < 0: r decreases along the trace */
                term = ORC_RAY_CAPTURED;
                tflag = ORC_FLAG_EARLY_CAPTURE;
                target = r_early;
            }
            if (term) {
                const double t = radius_crossing(y, yn, k, h, target);
                double yt[NB];
                dense(y, yn, k, h, t, yt);
                memcpy(y, yt, sizeof yt);
                lambda += t * h;
                status = term;
                flags |= tflag;
                break;
            }
        }
        dH = max_d(dH, project_null(c, yn, cam->projection_tol));
        reflect_pole(yn, k[6]);
        if (fm) { /* hydro model 2: the step's chord through the torus, L / E taken as
                   * u^phi r^2 sin^2(theta) at the step's end (:1529-1537) */
            double from[3], to[3];
            sph_cartesian(y, from);
            sph_cartesian(yn, to);
            const double st = sin(yn[1]);
            orc_fm_accumulate(fm, from, to, yn[6] * (yn[0] * yn[0] * st * st), vol);
        }
        lambda += h;
        memcpy(y, yn, sizeof yn);
        memcpy(k[0], k[6], sizeof(double) * NB);
        float factor = 5.0f;
        if (err != 0.0) {
            const float le = log2f(fmaxf((float)err, 1e-12f));
            factor = pi30f(le, has_hist ? ln_prev : le, 5.0f);
            ln_prev = le;
            has_hist = 1;
        }
        h = -clamp_d(fabs(h) * clamp_d(0.9 * factor, 0.2, 5.0), 1e-8, 1e13);
    }

    if (cont) {
        cont->fate = status;
        {
            /* the sky-lookup direction at the ray's end */
            double yr[7];
            memcpy(yr, y, sizeof yr);
            reflect_pole(yr, NULL);
            exit_direction(m, a, q2, yr, cont->exit_dir);
        }
        if (hit) {
            status = ORC_RAY_DISK;
            memcpy(y, y_hit, sizeof y_hit);
            lambda = lambda_hit;
            acc = acc_hit;
            rej = rej_hit;
            flags = flags_hit;
        }
    }
    reflect_pole(y, NULL);
    double iv[3];
    invariants(m, a, q2, y, iv);
    out->status = status;
    out->flags = flags;
    out->steps_accepted = acc;
    out->steps_rejected = rej;
    out->r = y[0];
    out->theta = y[1];
    out->phi = y[2];
    out->r_hit = r_hit;
    out->g = g;
    out->lambda = lambda;
    out->dH = dH;
    out->dE = iv[0] / E0 - 1.0;
    out->dLz = (iv[1] - inv0[1]) / E0;
    out->dQ = (iv[2] - inv0[2]) / (E0 * E0);
    out->db_shadow = db0;
    out->body = (status == ORC_RAY_DISK || status == ORC_RAY_CAPTURED) ? 0u : ORC_BODY_NONE;
    /* sky-lookup direction of an escaped ray (software_compute_engine.hpp:
     * 1581-1589 with local_frame_to_travel_direction, :1148-1168): the
     * orthonormal-frame velocity mapped to a Cartesian direction of travel */
    out->exit_dir[0] = out->exit_dir[1] = out->exit_dir[2] = NAN;
    if (status == ORC_RAY_ESCAPED) exit_direction(m, a, q2, y, out->exit_dir);
}

typedef struct {
    const orc_camera* cam;
    const bl_consts* c;
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
            trace_one(w->cam, w->c, (uint32_t)(pix % w->cam->screen_width), (uint32_t)(pix / w->cam->screen_width),
                      &w->out[i], w->cont ? &w->cont[i] : NULL, w->fm, w->vol ? w->vol + 6 * i : NULL);
        }
    }
    return NULL;
}

static void bl_trace_range(const orc_camera* cam, double charge, const uint64_t* pixel_index, uint64_t first,
                           uint64_t count, orc_ray* out, orc_cont* cont, const orc_fm* fm, double* vol,
                           int threads);

void orc_bl_trace(const orc_camera* cam, double charge, const uint64_t* pixel_index, uint64_t first, uint64_t count,
                  orc_ray* out, int threads)
{
    bl_trace_range(cam, charge, pixel_index, first, count, out, NULL, NULL, NULL, threads);
}

void orc_bl_trace_cont(const orc_camera* cam, double charge, const uint64_t* pixel_index, uint64_t first,
                       uint64_t count, orc_ray* out, orc_cont* cont, int threads)
{
    bl_trace_range(cam, charge, pixel_index, first, count, out, cont, NULL, NULL, threads);
}

void orc_bl_trace_volume(const orc_camera* cam, double charge, const orc_fm* fm, const uint64_t* pixel_index,
                         uint64_t first, uint64_t count, orc_ray* out, orc_cont* cont, double* vol, int threads)
{
    memset(vol, 0, sizeof(double) * 6 * count);
    bl_trace_range(cam, charge, pixel_index, first, count, out, cont, fm, vol, threads);
}

static void bl_trace_range(const orc_camera* cam, double charge, const uint64_t* pixel_index, uint64_t first,
                           uint64_t count, orc_ray* out, orc_cont* cont, const orc_fm* fm, double* vol,
                           int threads)
{
    bl_consts c;
    bl_camera_consts(cam, charge, &c);
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
