/*
 * ms_oracle.c -- FP64 CPU oracle of the multi-source Kerr-Schild tracer.
 *
 * TEST INFRASTRUCTURE ONLY (same rules as ks_oracle.c): a plain-C restatement
 * used as the checker of the CUDA multi-source kernel.
 *
 * What it restates (reference = Wartets/Relativity-Simulator,
 * include/relativistic/render/software_compute_engine.hpp):
 *   - source table: the camera's hole at the origin plus black-hole bodies, each
 *     with a local frame built from its spin axis   build_multi_source_data :2738-2798
 *   - superposed RHS: per-source Kerr-Schild terms in the local frame, summed in
 *     the world frame                                 ks_source_terms :2812-2855, ms_rhs :2857-2871
 *   - initial null momentum of a static observer in the superposed metric
 *                                                     ms_initial_momentum :2888-2964
 *   - inside-horizon test                             ms_inside_horizon :2966-2978
 *   - per-source disk crossing at local z = 0, r = sqrt(x^2 + y^2 - a^2), and
 *     g = redshift_at(m_i, a_i, r, L_z) with L_z from the unit local momentum
 *                                                     ms_disk_crossing :3023-3046, trace_multi_source :3155
 * The reference integrates this path with heuristic-step RK4; the oracle uses
 * the DP45 + PI30 + step cap machinery of ks_oracle.c, a step cap from the
 * nearest source, and a projection onto H = 0 of the superposed Hamiltonian
 * H = (|p|^2 - 1)/2 - sum_i H_i s_i^2 (s_i = 1 + k_i . p), whose Hamiltonian
 * flow is exactly the summed RHS.
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "ks_oracle.h"

#define ORC_PI 3.14159265358979323846

static inline double max_d(double a, double b) { return (a < b) ? b : a; }
static inline double min_d(double a, double b) { return (b < a) ? b : a; }
static inline double clamp_d(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
static inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* software_compute_engine.hpp:2738-2798 */
void orc_ms_build(const orc_camera* cam, const orc_source* src, uint32_t n, orc_ms_table* t)
{
    memset(t, 0, sizeof *t);
    const double m = max_d(cam->metric_mass, 1e-4);
    const double a = clamp_d(cam->metric_spin, -0.999 * m, 0.999 * m);
    const double rh = m + sqrt(max_d(m * m - a * a, 0.0));
    t->mass[0] = m;
    t->spin[0] = a;
    t->axis[0][2] = 1.0;
    t->fx[0][0] = 1.0;
    t->fy[0][1] = 1.0;
    t->rh[0] = rh;
    t->req[0] = sqrt(rh * rh + a * a);
    if (cam->disk_outer_radius > 0.0) {
        t->disk_in[0] = (cam->disk_inner_radius > 0.0) ? cam->disk_inner_radius : orc_isco_radius(m, a);
        t->disk_out[0] = cam->disk_outer_radius;
    } else {
        t->disk_in[0] = t->disk_out[0] = -1.0;
    }
    t->count = 1;
    for (uint32_t b = 0; b < n && t->count < ORC_MS_MAX_SOURCES; ++b) {
        const orc_source* s = &src[b];
        const uint32_t i = t->count;
        const double mb = max_d(s->mass, 1e-9);
        const double ab = clamp_d(s->spin_parameter, -0.9999, 0.9999) * mb;
        const double rhb = mb + sqrt(max_d(mb * mb - ab * ab, 0.0));
        const double len = sqrt(dot3(s->axis, s->axis));
        double axis[3] = {0.0, 0.0, 1.0};
        if (len > 1e-12)
            for (int k = 0; k < 3; ++k) axis[k] = s->axis[k] / len;
        const double helper[3] = {fabs(axis[2]) < 0.9 ? 0.0 : 1.0, 0.0, fabs(axis[2]) < 0.9 ? 1.0 : 0.0};
        double fx[3] = {helper[1] * axis[2] - helper[2] * axis[1], helper[2] * axis[0] - helper[0] * axis[2],
                        helper[0] * axis[1] - helper[1] * axis[0]};
        const double fl = sqrt(dot3(fx, fx));
        for (int k = 0; k < 3; ++k) fx[k] /= fl;
        const double fy[3] = {axis[1] * fx[2] - axis[2] * fx[1], axis[2] * fx[0] - axis[0] * fx[2],
                              axis[0] * fx[1] - axis[1] * fx[0]};
        for (int k = 0; k < 3; ++k) {
            t->pos[i][k] = s->position[k];
            t->axis[i][k] = axis[k];
            t->fx[i][k] = fx[k];
            t->fy[i][k] = fy[k];
        }
        t->mass[i] = mb;
        t->spin[i] = ab;
        t->rh[i] = rhb;
        t->req[i] = sqrt(rhb * rhb + ab * ab);
        if (s->disk_enabled > 0.5) {
            const double inner = orc_isco_radius(mb, ab) * max_d(s->disk_inner_scale, 1.0);
            t->disk_in[i] = inner;
            t->disk_out[i] = max_d(s->disk_outer_units * mb, inner * 1.05);
        } else {
            t->disk_in[i] = t->disk_out[i] = -1.0;
        }
        ++t->count;
    }
}

static inline void to_local(const orc_ms_table* t, uint32_t i, const double* d, double* l)
{
    l[0] = dot3(d, t->fx[i]);
    l[1] = dot3(d, t->fy[i]);
    l[2] = dot3(d, t->axis[i]);
}

static inline void to_world(const orc_ms_table* t, uint32_t i, const double* l, double* w)
{
    for (int k = 0; k < 3; ++k) w[k] = l[0] * t->fx[i][k] + l[1] * t->fy[i][k] + l[2] * t->axis[i][k];
}

/* Superposed RHS (ms_rhs :2857-2871).  Returns the step-cap length
 * min_i max(r_i - r_+i, 0.01 m_i) over the sources at y, and writes the index
 * of the first source whose local r_BL < scale * r_+ to *inside (-1: none). */
static double ms_rhs(const orc_ms_table* t, const double* y, double* dy, double capture_scale, int* inside)
{
    double cap = INFINITY;
    int in = -1;
    for (int k = 0; k < 3; ++k) {
        dy[k] = y[3 + k];
        dy[3 + k] = 0.0;
    }
    for (uint32_t i = 0; i < t->count; ++i) {
        const double rel[3] = {y[0] - t->pos[i][0], y[1] - t->pos[i][1], y[2] - t->pos[i][2]};
        double ly[6], ld[6];
        to_local(t, i, rel, ly);
        to_local(t, i, y + 3, ly + 3);
        double r, h, kk[3];
        orc_ks_field(ly, t->mass[i], t->spin[i], &r, &h, kk);
        orc_ks_rhs(ly, t->mass[i], t->spin[i], ld);
        /* the per-source position term is the gravitational part only */
        for (int k = 0; k < 3; ++k) ld[k] -= ly[3 + k];
        double w[3];
        to_world(t, i, ld, w);
        for (int k = 0; k < 3; ++k) dy[k] += w[k];
        to_world(t, i, ld + 3, w);
        for (int k = 0; k < 3; ++k) dy[3 + k] += w[k];
        cap = min_d(cap, max_d(r - t->rh[i], 0.01 * t->mass[i]));
        if (in < 0 && r < capture_scale * t->rh[i]) in = (int)i;
    }
    if (inside) *inside = in;
    return cap;
}

void orc_ms_rhs(const orc_ms_table* t, const double y[6], double dy[6]) { (void)ms_rhs(t, y, dy, 1.0, NULL); }

double orc_ms_hamiltonian(const orc_ms_table* t, const double y[6])
{
    double sum = 0.0;
    for (uint32_t i = 0; i < t->count; ++i) {
        const double rel[3] = {y[0] - t->pos[i][0], y[1] - t->pos[i][1], y[2] - t->pos[i][2]};
        double lx[3], lp[3], r, h, kk[3];
        to_local(t, i, rel, lx);
        to_local(t, i, y + 3, lp);
        orc_ks_field(lx, t->mass[i], t->spin[i], &r, &h, kk);
        const double s = 1.0 + dot3(kk, lp);
        sum += h * s * s;
    }
    return 0.5 * (dot3(y + 3, y + 3) - 1.0) - sum;
}

/* The superposed metric eta + 2 sum_i H_i l_i l_i on 4-vectors, l_i = (1, k_i)
 * (ms_metric_dot :2873-2886). */
static double ms_metric_dot(uint32_t n, const double* pot, double (*dir)[3], const double* a, const double* b)
{
    double v = -a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
    for (uint32_t i = 0; i < n; ++i) {
        const double la = a[0] + dir[i][0] * a[1] + dir[i][1] * a[2] + dir[i][2] * a[3];
        const double lb = b[0] + dir[i][0] * b[1] + dir[i][1] * b[2] + dir[i][2] * b[3];
        v += 2.0 * pot[i] * la * lb;
    }
    return v;
}

/* ms_initial_momentum :2888-2964: Gram-Schmidt of the coordinate axes lifted
 * into the static observer's rest space of the superposed metric, the null
 * vector u - outward, lowered and normalised to p_t = -1. */
void orc_ms_initial_momentum(const orc_ms_table* t, const double x[3], const double outward[3], double p[3])
{
    double pot[ORC_MS_MAX_SOURCES], dir[ORC_MS_MAX_SOURCES][3], sum = 0.0;
    for (uint32_t i = 0; i < t->count; ++i) {
        const double rel[3] = {x[0] - t->pos[i][0], x[1] - t->pos[i][1], x[2] - t->pos[i][2]};
        double lx[3], r, h, kk[3];
        to_local(t, i, rel, lx);
        orc_ks_field(lx, t->mass[i], t->spin[i], &r, &h, kk);
        pot[i] = h;
        to_world(t, i, kk, dir[i]);
        sum += h;
    }
    const double ilsq = 1.0 / max_d(1.0 - 2.0 * sum, 1e-6);
    const double u0 = sqrt(ilsq);
    double e[3][4];
    for (int j = 0; j < 3; ++j) { /* ms_lift of the coordinate axes */
        double v[3] = {0.0, 0.0, 0.0};
        v[j] = 1.0;
        double shift = 0.0;
        for (uint32_t i = 0; i < t->count; ++i) shift += pot[i] * dot3(dir[i], v);
        e[j][0] = 2.0 * shift * ilsq;
        e[j][1] = v[0];
        e[j][2] = v[1];
        e[j][3] = v[2];
    }
    /* Gram-Schmidt in the superposed metric; the projections of each axis on the
     * earlier ones are taken before any is subtracted, as the reference does */
    for (int j = 0; j < 3; ++j) {
        double d[2] = {0.0, 0.0};
        for (int q = 0; q < j; ++q) d[q] = ms_metric_dot(t->count, pot, dir, e[j], e[q]);
        for (int q = 0; q < j; ++q)
            for (int c = 0; c < 4; ++c) e[j][c] -= d[q] * e[q][c];
        const double norm = sqrt(max_d(ms_metric_dot(t->count, pot, dir, e[j], e[j]), 1e-30));
        for (int c = 0; c < 4; ++c) e[j][c] /= norm;
    }
    double v[4];
    for (int c = 0; c < 4; ++c) v[c] = -outward[0] * e[0][c] - outward[1] * e[1][c] - outward[2] * e[2][c];
    v[0] += u0;
    double mom[3] = {v[1], v[2], v[3]};
    double tc = -v[0];
    for (uint32_t i = 0; i < t->count; ++i) {
        const double lv = v[0] + dir[i][0] * v[1] + dir[i][1] * v[2] + dir[i][2] * v[3];
        tc += 2.0 * pot[i] * lv;
        for (int k = 0; k < 3; ++k) mom[k] += 2.0 * pot[i] * lv * dir[i][k];
    }
    const double inv = 1.0 / max_d(-tc, 1e-12);
    for (int k = 0; k < 3; ++k) p[k] = mom[k] * inv;
}

/* ms_inside_horizon :2966-2978 (with the reference's 1.0001 r_+ threshold). */
int orc_ms_inside_horizon(const orc_ms_table* t, const double x[3])
{
    for (uint32_t i = 0; i < t->count; ++i) {
        const double rel[3] = {x[0] - t->pos[i][0], x[1] - t->pos[i][1], x[2] - t->pos[i][2]};
        double l[3];
        to_local(t, i, rel, l);
        const double a2 = t->spin[i] * t->spin[i];
        const double diff = dot3(l, l) - a2;
        const double r2 = max_d(0.5 * (diff + sqrt(diff * diff + 4.0 * a2 * l[2] * l[2])), 1e-24);
        const double r = sqrt(r2);
        if (r <= t->rh[i] * 1.0001 || (r2 - 2.0 * t->mass[i] * r + a2) <= 0.0) return 1;
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* DP45 on the superposed RHS (tableau as ks_oracle.c, rk45_adaptive.hpp:196-261). */
static const double A21 = 1.0 / 5.0;
static const double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
static const double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
static const double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0, A54 = -212.0 / 729.0;
static const double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0, A64 = 49.0 / 176.0,
                    A65 = -5103.0 / 18656.0;
static const double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0, B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
static const double E1 = 71.0 / 57600.0, E3 = -71.0 / 16695.0, E4 = 71.0 / 1920.0, E5 = -17253.0 / 339200.0,
                    E6 = 22.0 / 525.0, E7 = -1.0 / 40.0;
/* continuous extension of order 4 (Hairer, Norsett & Wanner, sec. II.6) */
static const double D1 = -12715105075.0 / 11282082432.0, D3 = 87487479700.0 / 32700410799.0,
                    D4 = -10690763975.0 / 1880347072.0, D5 = 701980252875.0 / 199316789632.0,
                    D6 = -1453857185.0 / 822651844.0, D7 = 69997945.0 / 29380423.0;

static void stages(const orc_ms_table* t, const double* y, double h, double k[7][6], double* y5)
{
    double s[6];
    for (int i = 0; i < 6; ++i) s[i] = y[i] + h * (A21 * k[0][i]);
    ms_rhs(t, s, k[1], 1.0, NULL);
    for (int i = 0; i < 6; ++i) s[i] = y[i] + h * (A31 * k[0][i] + A32 * k[1][i]);
    ms_rhs(t, s, k[2], 1.0, NULL);
    for (int i = 0; i < 6; ++i) s[i] = y[i] + h * (A41 * k[0][i] + A42 * k[1][i] + A43 * k[2][i]);
    ms_rhs(t, s, k[3], 1.0, NULL);
    for (int i = 0; i < 6; ++i) s[i] = y[i] + h * (A51 * k[0][i] + A52 * k[1][i] + A53 * k[2][i] + A54 * k[3][i]);
    ms_rhs(t, s, k[4], 1.0, NULL);
    for (int i = 0; i < 6; ++i)
        s[i] = y[i] + h * (A61 * k[0][i] + A62 * k[1][i] + A63 * k[2][i] + A64 * k[3][i] + A65 * k[4][i]);
    ms_rhs(t, s, k[5], 1.0, NULL);
    for (int i = 0; i < 6; ++i)
        y5[i] = y[i] + h * (B1 * k[0][i] + B3 * k[2][i] + B4 * k[3][i] + B5 * k[4][i] + B6 * k[5][i]);
}

/* Dense output y(theta) of an accepted step. */
static void dense(const double* y0, const double* y1, double k[7][6], double h, double th, double* out)
{
    for (int i = 0; i < 6; ++i) {
        const double d = y1[i] - y0[i];
        const double b = h * k[0][i] - d;
        const double c = d - h * k[6][i] - b;
        const double e = h * (D1 * k[0][i] + D3 * k[2][i] + D4 * k[3][i] + D5 * k[4][i] + D6 * k[5][i] + D7 * k[6][i]);
        out[i] = y0[i] + th * (d + (1.0 - th) * (b + th * (c + (1.0 - th) * e)));
    }
}

/* Illinois root on [0, 1] of f(theta) = axis . (y(theta) - pos) (local z of source i). */
static double local_z_root(const orc_ms_table* t, uint32_t i, const double* y0, const double* y1, double k[7][6],
                           double h, double f0, double f1)
{
    double lo = 0.0, hi = 1.0, flo = f0, fhi = f1, th = 1.0, yy[6];
    int side = 0;
    for (int it = 0; it < 60; ++it) {
        th = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(th > lo && th < hi)) th = 0.5 * (lo + hi);
        dense(y0, y1, k, h, th, yy);
        const double rel[3] = {yy[0] - t->pos[i][0], yy[1] - t->pos[i][1], yy[2] - t->pos[i][2]};
        const double ft = dot3(rel, t->axis[i]);
        if (ft == 0.0 || fabs(hi - lo) < 1e-15 || fabs(ft) < 1e-13 * (1.0 + fabs(rel[0]) + fabs(rel[1]))) break;
        if ((ft > 0.0) == (fhi > 0.0)) {
            hi = th;
            fhi = ft;
            if (side == -1) flo *= 0.5;
            side = -1;
        } else {
            lo = th;
            flo = ft;
            if (side == 1) fhi *= 0.5;
            side = 1;
        }
    }
    return th;
}

/* Cubic Hermite interpolant on the FSAL end points, and the fraction where
 * |x| crosses the escape radius (Illinois). */
static void hermite(const double* y0, const double* f0, const double* y1, const double* f1, double h, double t, double* out)
{
    const double t2 = t * t, t3 = t2 * t;
    const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + t, h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
    for (int i = 0; i < 6; ++i) out[i] = h00 * y0[i] + h10 * h * f0[i] + h01 * y1[i] + h11 * h * f1[i];
}

static double radius_crossing(const double* y0, const double* f0, const double* y1, const double* f1, double h,
                              double target)
{
    double lo = 0.0, hi = 1.0, x[6];
    double flo = sqrt(dot3(y0, y0)) - target, fhi = sqrt(dot3(y1, y1)) - target;
    if (!((flo > 0.0) != (fhi > 0.0))) return 1.0;
    int side = 0;
    double t = 1.0;
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        hermite(y0, f0, y1, f1, h, t, x);
        const double ft = sqrt(dot3(x, x)) - target;
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

/* Projection of p onto H = 0 along n = dH/dp (closest root), H the superposed Hamiltonian. */
static double project_ms(const orc_ms_table* t, double* y, double tol)
{
    double* p = y + 3;
    double n[3] = {p[0], p[1], p[2]};
    double hs[ORC_MS_MAX_SOURCES], s[ORC_MS_MAX_SOURCES], kw[ORC_MS_MAX_SOURCES][3];
    double sum = 0.0;
    for (uint32_t i = 0; i < t->count; ++i) {
        const double rel[3] = {y[0] - t->pos[i][0], y[1] - t->pos[i][1], y[2] - t->pos[i][2]};
        double lx[3], r, h, kl[3];
        to_local(t, i, rel, lx);
        orc_ks_field(lx, t->mass[i], t->spin[i], &r, &h, kl);
        to_world(t, i, kl, kw[i]);
        s[i] = 1.0 + dot3(kw[i], p);
        hs[i] = h;
        sum += h * s[i] * s[i];
        for (int k = 0; k < 3; ++k) n[k] -= 2.0 * h * s[i] * kw[i][k];
    }
    const double res = 0.5 * (dot3(p, p) - 1.0) - sum;
    if (!(fabs(res) >= tol)) return fabs(res);
    double qa = 0.5 * dot3(n, n), qb = dot3(p, n);
    for (uint32_t i = 0; i < t->count; ++i) {
        const double kn = dot3(kw[i], n);
        qa -= hs[i] * kn * kn;
        qb -= 2.0 * hs[i] * s[i] * kn;
    }
    const double disc = qb * qb - 4.0 * qa * res;
    if (disc >= 0.0) {
        const double q = -0.5 * (qb + copysign(sqrt(disc), qb));
        if (q != 0.0) {
            const double alpha = res / q;
            for (int k = 0; k < 3; ++k) p[k] += alpha * n[k];
        }
    }
    return fabs(res);
}

static inline float pi30f(float le, float lp, float order_p1)
{
    return exp2f(-(0.7f / order_p1) * le + (0.3f / order_p1) * (lp - le));
}

/* Initial state of pixel (px, py): the observer at the Cartesian point of
 * (r, theta, phi) and the pinhole ray's world direction as `outward`
 * (trace_multi_source :3049-3068). */
void orc_ms_initial_state(const orc_camera* cam, const orc_ms_table* t, uint32_t px, uint32_t py, double y0[6])
{
    const double W = (double)cam->screen_width, H = (double)cam->screen_height;
    const double v = 1.0 - ((double)py + 0.5) / H * 2.0;
    const double u = (((double)px + 0.5) / W * 2.0 - 1.0) * (W / H);
    double n[3];
    orc_pinhole_ray(u, v, cam->field_of_view_rad, n);
    double d[3];
    for (int i = 0; i < 3; ++i)
        d[i] = n[0] * cam->tetrad_e1[1 + i] + n[2] * cam->tetrad_e2[1 + i] + n[1] * cam->tetrad_e3[1 + i];
    const double r = cam->observer_position[1];
    const double th = clamp_d(cam->observer_position[2], 0.001, ORC_PI - 0.001), ph = cam->observer_position[3];
    y0[0] = r * sin(th) * cos(ph);
    y0[1] = r * sin(th) * sin(ph);
    y0[2] = r * cos(th);
    orc_ms_initial_momentum(t, y0, d, y0 + 3);
}

static inline void unwrap_to(double* phi, const double* y)
{
    double d = atan2(y[1], y[0]) - *phi;
    d -= 2.0 * ORC_PI * floor(d / (2.0 * ORC_PI) + 0.5);
    *phi += d;
}

/* One ray; with `cont`, the translucent-disk continuation (crossings recorded
 * in order along the ray, the record describing the first hit). */
static void trace_one(const orc_camera* cam, const orc_ms_table* t, uint32_t px, uint32_t py, orc_ray* out,
                      orc_cont* cont)
{
    double y[6];
    orc_ms_initial_state(cam, t, px, py, y);
    double k[7][6];
    int inside;
    double cap_len = ms_rhs(t, y, k[0], cam->capture_scale, &inside);
    double h = -cam->initial_step_fraction * cam->observer_position[1];
    double lambda = 0.0, dH = 0.0, r_hit = NAN, g = 1.0;
    float ln_prev = 0.0f;
    int has_hist = 0;
    uint32_t acc = 0, rej = 0, status = ORC_RAY_UNFINISHED, flags = 0;
    double phi = atan2(y[1], y[0]);
    double yn[6];
    uint32_t body = ORC_BODY_NONE;
    /* continuation: the first hit's record */
    int hit = 0;
    double y_hit[6], lambda_hit = 0.0, phi_hit = 0.0, r_hit1 = NAN, g_hit1 = 1.0;
    uint32_t acc_hit = 0, rej_hit = 0, flags_hit = 0, body_hit = 0;
    if (cont) {
        memset(cont, 0, sizeof *cont);
        cont->fate = ORC_RAY_UNFINISHED;
        cont->exit_dir[0] = cont->exit_dir[1] = cont->exit_dir[2] = NAN;
    }
    for (uint32_t attempt = 0;; ++attempt) {
        if (inside >= 0) {
            status = ORC_RAY_CAPTURED;
            body = (uint32_t)inside;
            break;
        }
        if (dot3(y + 3, y + 3) > ORC_MS_MAX_MOMENTUM * ORC_MS_MAX_MOMENTUM) {
            status = ORC_RAY_CAPTURED;
            flags |= ORC_FLAG_DIVERGED;
            break;
        }
        if (sqrt(dot3(y, y)) > cam->escape_radius) {
            status = ORC_RAY_ESCAPED;
            break;
        }
        if (attempt >= cam->max_steps) {
            flags |= ORC_FLAG_MAX_STEPS;
            break;
        }
        const double cap = cam->step_cap_fraction * cap_len;
        if (fabs(h) > cap) h = -cap;
        if (fabs(h) < 1e-8) {
            status = ORC_RAY_CAPTURED;
            flags |= ORC_FLAG_STEP_UNDERFLOW;
            break;
        }
        stages(t, y, h, k, yn);
        int inside_n;
        const double cap_n = ms_rhs(t, yn, k[6], cam->capture_scale, &inside_n);
        double err = 0.0;
        for (int i = 0; i < 6; ++i) {
            const double est = fabs(h) * fabs(E1 * k[0][i] + E3 * k[2][i] + E4 * k[3][i] + E5 * k[4][i] +
                                            E6 * k[5][i] + E7 * k[6][i]);
            err = max_d(err, est / (cam->rtol * max_d(fabs(y[i]), fabs(yn[i])) + cam->atol));
        }
        if (!(err <= 1e300)) err = 1e300;
        if (err <= 1.0) {
            ++acc;
            int nonfinite = 0;
            for (int i = 0; i < 6; ++i) nonfinite |= !isfinite(yn[i]);
            if (nonfinite) {
                status = ORC_RAY_CAPTURED;
                flags |= ORC_FLAG_NONFINITE;
                break;
            }
            /* disk crossings of the step in order along the ray: the earliest
             * local z = 0 root on a disk after the previous one */
            int ended = 0;
            double t_prev = -1.0;
            for (uint32_t pass = 0; pass < t->count; ++pass) {
                double best = 2.0, best_r = 0.0, best_g = 1.0, best_az = 0.0, best_y[6];
                uint32_t best_i = 0;
                for (uint32_t i = 0; i < t->count; ++i) {
                    if (t->disk_in[i] < 0.0) continue;
                    const double r0[3] = {y[0] - t->pos[i][0], y[1] - t->pos[i][1], y[2] - t->pos[i][2]};
                    const double r1[3] = {yn[0] - t->pos[i][0], yn[1] - t->pos[i][1], yn[2] - t->pos[i][2]};
                    const double z0 = dot3(r0, t->axis[i]), z1 = dot3(r1, t->axis[i]);
                    if (!(z0 * z1 <= 0.0) || z0 == z1) continue;
                    /* linear estimate with a margin before the root solve */
                    const double sl = z0 / (z0 - z1);
                    double ce[3], le[3];
                    for (int q = 0; q < 3; ++q) ce[q] = r0[q] + sl * (r1[q] - r0[q]);
                    to_local(t, i, ce, le);
                    const double a = t->spin[i];
                    const double re = sqrt(max_d(le[0] * le[0] + le[1] * le[1] - a * a, 0.0));
                    const double margin = 0.05 * re + 0.5 * t->mass[i];
                    if (re < t->disk_in[i] - margin || re > t->disk_out[i] + margin) continue;
                    const double th = local_z_root(t, i, y, yn, k, h, z0, z1);
                    if (!(th < best) || !(th > t_prev)) continue;
                    double yr[6];
                    dense(y, yn, k, h, th, yr);
                    const double rel[3] = {yr[0] - t->pos[i][0], yr[1] - t->pos[i][1], yr[2] - t->pos[i][2]};
                    double c[3], pl[3];
                    to_local(t, i, rel, c);
                    to_local(t, i, yr + 3, pl);
                    const double rr = sqrt(max_d(c[0] * c[0] + c[1] * c[1] - a * a, 0.0));
                    if (rr < t->disk_in[i] || rr > t->disk_out[i] || rr <= t->rh[i] * 1.02) continue;
                    const double lz = (c[0] * pl[1] - c[1] * pl[0]) / max_d(sqrt(dot3(pl, pl)), 1e-30);
                    best = th;
                    best_r = rr;
                    best_g = orc_redshift_at(t->mass[i], a, rr, lz);
                    /* local azimuth of the crossing (ms_disk_crossing, software_compute_engine.hpp:3037) */
                    best_az = atan2(c[1], c[0]) - atan2(a, rr);
                    best_i = i;
                    memcpy(best_y, yr, sizeof yr);
                }
                if (best > 1.0) break;
                if (!cont) {
                    status = ORC_RAY_DISK;
                    body = best_i;
                    r_hit = best_r;
                    g = best_g;
                    lambda += best * h;
                    unwrap_to(&phi, best_y);
                    memcpy(y, best_y, sizeof best_y);
                    ended = 1;
                    break;
                }
                const uint32_t kx = cont->n_cross++;
                cont->cross_r[kx] = best_r;
                cont->cross_phi[kx] = best_az;
                cont->cross_g[kx] = best_g;
                cont->cross_src[kx] = best_i;
                if (!hit) {
                    hit = 1;
                    memcpy(y_hit, best_y, sizeof best_y);
                    lambda_hit = lambda + best * h;
                    phi_hit = phi;
                    unwrap_to(&phi_hit, best_y);
                    r_hit1 = best_r;
                    g_hit1 = best_g;
                    acc_hit = acc;
                    rej_hit = rej;
                    flags_hit = flags;
                    body_hit = best_i;
                }
                t_prev = best;
                if (cont->n_cross >= ORC_MAX_CROSSINGS) {
                    memcpy(y, best_y, sizeof best_y);
                    ended = 1;
                    break;
                }
            }
            if (ended) break;
            if (inside_n >= 0) { /* captured inside this step: the end point */
                lambda += h;
                {
                    double d = atan2(yn[1], yn[0]) - phi;
                    d -= 2.0 * ORC_PI * floor(d / (2.0 * ORC_PI) + 0.5);
                    phi += d;
                }
                memcpy(y, yn, sizeof yn);
                status = ORC_RAY_CAPTURED;
                body = (uint32_t)inside_n;
                break;
            }
            if (sqrt(dot3(yn, yn)) > cam->escape_radius) { /* escaped: interpolated to the escape radius */
                const double tt = radius_crossing(y, k[0], yn, k[6], h, cam->escape_radius);
                double yt[6];
                hermite(y, k[0], yn, k[6], h, tt, yt);
                lambda += tt * h;
                {
                    double d = atan2(yt[1], yt[0]) - phi;
                    d -= 2.0 * ORC_PI * floor(d / (2.0 * ORC_PI) + 0.5);
                    phi += d;
                }
                memcpy(y, yt, sizeof yt);
                status = ORC_RAY_ESCAPED;
                break;
            }
            dH = max_d(dH, project_ms(t, yn, cam->projection_tol));
            {
                double d = atan2(yn[1], yn[0]) - phi;
                d -= 2.0 * ORC_PI * floor(d / (2.0 * ORC_PI) + 0.5);
                phi += d;
            }
            lambda += h;
            memcpy(y, yn, sizeof yn);
            memcpy(k[0], k[6], sizeof(double) * 6);
            cap_len = cap_n;
            inside = inside_n;
            float factor = 5.0f;
            if (err != 0.0) {
                const float le = log2f(fmaxf((float)err, 1e-12f));
                factor = pi30f(le, has_hist ? ln_prev : le, 5.0f);
                ln_prev = le;
                has_hist = 1;
            }
            h = -clamp_d(fabs(h) * clamp_d(0.9 * factor, 0.2, 5.0), 1e-8, 1e13);
        } else {
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
        cont->near_source = 0;
        for (uint32_t i = 0; i < t->count; ++i) {
            const double d[3] = {y[0] - t->pos[i][0], y[1] - t->pos[i][1], y[2] - t->pos[i][2]};
            if (sqrt(dot3(d, d)) < 6.0 * t->mass[i]) cont->near_source = 1;
        }
        {  /* the sky-lookup direction at the ray's end */
            double dy[6];
            orc_ms_rhs(t, y, dy);
            const double len = sqrt(dy[0] * dy[0] + dy[1] * dy[1] + dy[2] * dy[2]);
            if (len > 1e-12) {
                for (int i = 0; i < 3; ++i) cont->exit_dir[i] = -dy[i] / len;
            } else {
                cont->exit_dir[0] = cont->exit_dir[1] = 0.0;
                cont->exit_dir[2] = -1.0;
            }
        }
        if (hit) {
            /* the record describes the first hit */
            status = ORC_RAY_DISK;
            memcpy(y, y_hit, sizeof y_hit);
            lambda = lambda_hit;
            phi = phi_hit;
            r_hit = r_hit1;
            g = g_hit1;
            acc = acc_hit;
            rej = rej_hit;
            flags = flags_hit;
            body = body_hit;
        }
    }
    const double rr = sqrt(dot3(y, y));
    out->body = body;
    out->status = status;
    out->flags = flags;
    out->steps_accepted = acc;
    out->steps_rejected = rej;
    out->r = rr;
    out->theta = acos(clamp_d(y[2] / max_d(rr, 1e-300), -1.0, 1.0));
    out->phi = phi;
    out->r_hit = r_hit;
    out->g = g;
    out->lambda = lambda;
    out->dH = dH;
    out->dE = NAN;
    out->dLz = NAN;
    out->dQ = NAN;
    out->db_shadow = NAN;
    /* sky-lookup direction of an escaped ray: minus the normalised flow of the
     * superposed RHS at the terminal state, (0, 0, -1) where it vanishes
     * (software_compute_engine.hpp:3220-3224) */
    out->exit_dir[0] = out->exit_dir[1] = out->exit_dir[2] = NAN;
    if (status == ORC_RAY_ESCAPED) {
        double dy[6];
        orc_ms_rhs(t, y, dy);
        const double len = sqrt(dy[0] * dy[0] + dy[1] * dy[1] + dy[2] * dy[2]);
        if (len > 1e-12) {
            for (int i = 0; i < 3; ++i) out->exit_dir[i] = -dy[i] / len;
        } else {
            out->exit_dir[0] = out->exit_dir[1] = 0.0;
            out->exit_dir[2] = -1.0;
        }
    }
}

typedef struct {
    const orc_camera* cam;
    const orc_ms_table* t;
    const uint64_t* idx;
    uint64_t first, count;
    orc_ray* out;
    orc_cont* cont;
    atomic_ullong next;
} work_t;

static void* worker(void* arg)
{
    work_t* w = (work_t*)arg;
    for (;;) {
        const uint64_t b = atomic_fetch_add(&w->next, 8);
        if (b >= w->count) break;
        const uint64_t e = (b + 8 < w->count) ? b + 8 : w->count;
        for (uint64_t i = b; i < e; ++i) {
            const uint64_t pix = w->idx ? w->idx[i] : w->first + i;
            trace_one(w->cam, w->t, (uint32_t)(pix % w->cam->screen_width), (uint32_t)(pix / w->cam->screen_width),
                      &w->out[i], w->cont ? &w->cont[i] : NULL);
        }
    }
    return NULL;
}

static void run(const orc_camera* cam, const orc_ms_table* t, const uint64_t* pixel_index, uint64_t first,
                uint64_t count, orc_ray* out, orc_cont* cont, int threads)
{
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    work_t w;
    w.cam = cam;
    w.t = t;
    w.idx = pixel_index;
    w.first = first;
    w.count = count;
    w.out = out;
    w.cont = cont;
    atomic_init(&w.next, 0);
    pthread_t* tid = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    int started = 0;
    for (int i = 0; threads > 1 && i < threads; ++i)
        if (pthread_create(&tid[i], NULL, worker, &w) == 0) ++started;
    if (started == 0) worker(&w);
    for (int i = 0; i < started; ++i) pthread_join(tid[i], NULL);
    free(tid);
}

void orc_ms_trace(const orc_camera* cam, const orc_ms_table* t, const uint64_t* pixel_index, uint64_t first,
                  uint64_t count, orc_ray* out, int threads)
{
    run(cam, t, pixel_index, first, count, out, NULL, threads);
}

void orc_ms_trace_cont(const orc_camera* cam, const orc_ms_table* t, const uint64_t* pixel_index, uint64_t first,
                       uint64_t count, orc_ray* out, orc_cont* cont, int threads)
{
    run(cam, t, pixel_index, first, count, out, cont, threads);
}
