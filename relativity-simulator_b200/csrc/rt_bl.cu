// rt_bl.cu -- Boyer-Lindquist Kerr-Newman tracer for sm_100a (FP64).
//
// The engine's exact-metric path for black holes with charge (metric type 5,
// KerrNewmanMetric) and for Boyer-Lindquist Kerr / Schwarzschild cameras
// (SoftwareComputeEngine::trace_exact_photon, software_compute_engine.hpp:
// 1334-1622, routed by trace_exact_photon_dispatch :3364-3391).  Per ray:
//   - the ZAMO light ray u = e0 - n^i e_i at the observer (:1347-1350,
//     observer_tetrad.hpp:82-100, 144-166);
//   - the geodesic equation du/dl = -Gamma^mu_ab u^a u^b (rk45_adaptive.hpp:
//     64-88) on y = (r, theta, phi, u^t, u^r, u^theta, u^phi), contracted in
//     factored form from the r- and theta-derivatives of the five metric
//     components (kerr_newman.hpp:203-251) instead of forming 40 symbols;
//   - Dormand-Prince 5(4) with PI30 control, the step cap
//     |h| <= c max(r - r_+, 0.01 M), and after each accepted step the null
//     condition solved for u^t, root closest to the current u^t
//     (rk45_adaptive.hpp:91-139), then the pole reflection (:1492-1500);
//   - classification: captured (r < capture_scale r_+), escaped, disk (first
//     theta = pi/2 crossing with r on [r_in, r_out] and r > 1.02 r_+, :1538-1547,
//     root on the step's dense output, g = redshift_at(M, a, r, L/E)), and the
//     certain-capture early-out with the Kerr-Newman radial potential.
// Terminal points are placed on the step's dense output at the threshold
// radius.  The heuristic RK4 of the reference is replaced by the adaptive
// step, as in the Kerr-Schild tracer.  The stage loop is rolled around one
// copy of the right-hand side; stage derivatives k2..k7 live in shared memory.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "rt_device.cuh"
#include "rt_internal.h"
#include "rt_shade.cuh"

namespace relsim {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kHalfPi = 0.5 * kPi;
constexpr double kEarlyCaptureMargin = 1e-4;  // M, distance to the critical curve
constexpr int NB = 7;
enum BlMode : int { BL_IDLE = 0, BL_STEP = 1 };

// Dormand-Prince rows (rk45_adaptive.hpp:196-203), error and dense-output weights.
__constant__ double kBlA[6][6] = {
    {DP::A21, 0, 0, 0, 0, 0},
    {DP::A31, DP::A32, 0, 0, 0, 0},
    {DP::A41, DP::A42, DP::A43, 0, 0, 0},
    {DP::A51, DP::A52, DP::A53, DP::A54, 0, 0},
    {DP::A61, DP::A62, DP::A63, DP::A64, DP::A65, 0},
    {DP::B1, 0.0, DP::B3, DP::B4, DP::B5, DP::B6}};
__constant__ double kBlE[7] = {DP::E1, 0.0, DP::E3, DP::E4, DP::E5, DP::E6, DP::E7};
__constant__ double kBlD[7] = {DP::D1, 0.0, DP::D3, DP::D4, DP::D5, DP::D6, DP::D7};

template <int BLOCK>
struct BlCold {
    double k[6][NB][BLOCK];  // stage derivatives k2..k7
    double lambda[BLOCK];
    double dH[BLOCK];
    double e0[BLOCK], l0[BLOCK], q0[BLOCK];  // E, L, Carter Q at the observer
    uint64_t local[BLOCK];
};

// Metric components (g_tt, g_tphi, g_rr, g_thth, g_phiphi) at (r, theta) and,
// with DERIV, their r- and theta-derivatives.  F = (2 M r - Q^2) / rho^2:
//   g_tt = F - 1, g_tphi = -a s^2 F, g_rr = rho^2 / Delta, g_thth = rho^2,
//   g_phiphi = s^2 (r^2 + a^2 + a^2 s^2 F).
// One reciprocal of rho^2 Delta max(s^2, 1e-30) gives 1/rho^2, 1/Delta,
// 1/g_rr and 1/(Delta s^2) (the t-phi block's determinant is -Delta s^2).
struct KnGeom {
    double g[5], dr[5], dth[5];
    double irho2, idelta, idet, grr_inv, sin2, cos1;
};

template <bool DERIV>
__device__ __forceinline__ void kn_geometry(double m, double a, double q2, double r, double th, KnGeom& G) {
    double s, c;
    sincos(th, &s, &c);
    const double s2 = s * s, sc = s * c;
    const double a2 = a * a, r2 = r * r;
    const double rho2 = r2 + a2 * (c * c);
    const double delta = r2 - 2.0 * m * r + a2 + q2;
    const double s2c = fmax(s2, 1e-30);
    const double qinv = 1.0 / (rho2 * delta * s2c);
    const double irho2 = delta * s2c * qinv;
    const double idelta = rho2 * s2c * qinv;
    const double F = (2.0 * m * r - q2) * irho2;
    const double W = r2 + a2 + a2 * s2 * F;
    G.g[0] = F - 1.0;
    G.g[1] = -a * s2 * F;
    G.g[2] = rho2 * idelta;
    G.g[3] = rho2;
    G.g[4] = s2 * W;
    G.irho2 = irho2;
    G.idelta = idelta;
    G.idet = -rho2 * qinv;
    G.grr_inv = delta * irho2;
    G.sin2 = s2c;
    G.cos1 = c;
    if constexpr (DERIV) {
        const double dFr = (2.0 * m - 2.0 * r * F) * irho2;
        const double dFt = 2.0 * a2 * sc * F * irho2;
        const double sF = 2.0 * sc * F + s2 * dFt;
        G.dr[0] = dFr;
        G.dr[1] = -a * s2 * dFr;
        G.dr[2] = (2.0 * r - G.g[2] * (2.0 * r - 2.0 * m)) * idelta;
        G.dr[3] = 2.0 * r;
        G.dr[4] = s2 * (2.0 * r + a2 * s2 * dFr);
        G.dth[0] = dFt;
        G.dth[1] = -a * sF;
        G.dth[2] = -2.0 * a2 * sc * idelta;
        G.dth[3] = -2.0 * a2 * sc;
        G.dth[4] = 2.0 * sc * W + s2 * a2 * sF;
    }
}

// du/dl = -Gamma u u from d(g_mu nu u^nu)/dl = (1/2) d_mu g_ab u^a u^b:
//   r, theta: g_rr a^r = (1/2) d_r g(u,u) - (d_r g_rr u^r + d_th g_rr u^th) u^r (same for theta);
//   t, phi:   the t-phi block times (a^t, a^phi) = -(dg/dl) (u^t, u^phi).
__device__ __forceinline__ void bl_rhs(double m, double a, double q2, const double* __restrict__ y,
                                       double* __restrict__ dy) {
    KnGeom G;
    kn_geometry<true>(m, a, q2, y[0], y[1], G);
    const double ut = y[3], ur = y[4], uth = y[5], up = y[6];
    const double half_r = 0.5 * (G.dr[0] * ut * ut + 2.0 * G.dr[1] * ut * up + G.dr[2] * ur * ur +
                                 G.dr[3] * uth * uth + G.dr[4] * up * up);
    const double half_t = 0.5 * (G.dth[0] * ut * ut + 2.0 * G.dth[1] * ut * up + G.dth[2] * ur * ur +
                                 G.dth[3] * uth * uth + G.dth[4] * up * up);
    const double dgtt = G.dr[0] * ur + G.dth[0] * uth;
    const double dgtp = G.dr[1] * ur + G.dth[1] * uth;
    const double dgpp = G.dr[4] * ur + G.dth[4] * uth;
    const double bt = -(dgtt * ut + dgtp * up);
    const double bp = -(dgtp * ut + dgpp * up);
    dy[0] = ur;
    dy[1] = uth;
    dy[2] = up;
    dy[3] = (G.g[4] * bt - G.g[1] * bp) * G.idet;
    dy[4] = (half_r - (G.dr[2] * ur + G.dth[2] * uth) * ur) * G.grr_inv;
    dy[5] = (half_t - (G.dr[3] * ur + G.dth[3] * uth) * uth) * G.irho2;
    dy[6] = (G.g[0] * bp - G.g[1] * bt) * G.idet;
}

// Stages 2..7 around one RHS copy; S.k holds k2..k7 on return (k7 = S.k[5]).
// Returns the max-norm error (rk45_adaptive.hpp:254-261, with |h|).
template <int BLOCK>
__device__ __forceinline__ double bl_stages(const BlDesc& B, const double* __restrict__ y,
                                            const double* __restrict__ k1, double hh, BlCold<BLOCK>& S, int tid,
                                            double* __restrict__ y5) {
#pragma unroll
    for (int st = 0; st < 6; ++st) {
        double in[NB];
        // the stage sum unrolled over j (predicated on j <= st): every shared-memory
        // load of the stage is independent of the others and issues up front
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            double acc = kBlA[st][0] * k1[i];
#pragma unroll
            for (int j = 1; j < 6; ++j)
                if (j <= st) acc += kBlA[st][j] * S.k[j - 1][i][tid];
            in[i] = y[i] + hh * acc;
        }
        if (st == 5) {
#pragma unroll
            for (int i = 0; i < NB; ++i) y5[i] = in[i];
        }
        double out[NB];
        bl_rhs(B.m, B.a, B.q2, in, out);
#pragma unroll
        for (int i = 0; i < NB; ++i) S.k[st][i][tid] = out[i];
    }
    double num = 0.0, den = 1.0;
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        double acc = kBlE[0] * k1[i];
#pragma unroll
        for (int j = 2; j < 7; ++j) acc += kBlE[j] * S.k[j - 1][i][tid];
        const double est = fabs(hh) * fabs(acc);
        const double sc = B.rtol * fmax(fabs(y[i]), fabs(y5[i])) + B.atol;
        if (est * den > num * sc) {
            num = est;
            den = sc;
        }
    }
    return num / den;
}

// Dense output y(t) = y0 + t (d + (1-t)(b + t(c + (1-t) e))) of the accepted step.
template <int BLOCK>
__device__ __forceinline__ void bl_dense_coeffs(const double* __restrict__ y0, const double* __restrict__ y1,
                                                const double* __restrict__ k1, const double* __restrict__ k7,
                                                double h, const BlCold<BLOCK>& S, int tid, double (*co)[NB]) {
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const double d = y1[i] - y0[i];
        const double b = h * k1[i] - d;
        double e = kBlD[0] * k1[i] + kBlD[6] * k7[i];
#pragma unroll 1
        for (int j = 2; j < 6; ++j) e += kBlD[j] * S.k[j - 1][i][tid];
        co[0][i] = d;
        co[1][i] = b;
        co[2][i] = d - h * k7[i] - b;
        co[3][i] = h * e;
    }
}

__device__ __forceinline__ double bl_dense_at(const double* y0, const double (*co)[NB], int i, double t) {
    return y0[i] + t * (co[0][i] + (1.0 - t) * (co[1][i] + t * (co[2][i] + (1.0 - t) * co[3][i])));
}

// Illinois root on [0, 1] of component i of the dense output minus target.
__device__ double bl_dense_root(const double* y0, const double (*co)[NB], int i, double target, double f0, double f1,
                                double ftol) {
    double lo = 0.0, hi = 1.0, flo = f0, fhi = f1, t = 1.0;
    int side = 0;
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        const double ft = bl_dense_at(y0, co, i, t) - target;
        if (ft == 0.0 || fabs(hi - lo) < 1e-15 || fabs(ft) < ftol) break;
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

// u^t <- the root of g(u, u) = 0 closest to the current u^t (cancellation-free
// pair q / A, C / q); returns |(1/2) g(u, u)| before.
__device__ __forceinline__ double bl_project(const BlDesc& B, double* y) {
    KnGeom G;
    kn_geometry<false>(B.m, B.a, B.q2, y[0], y[1], G);
    const double ut = y[3], ur = y[4], uth = y[5], up = y[6];
    const double A = G.g[0];
    const double Bq = 2.0 * G.g[1] * up;
    const double C = G.g[2] * ur * ur + G.g[3] * uth * uth + G.g[4] * up * up;
    const double res = 0.5 * ((A * ut + Bq) * ut + C);
    if (!(fabs(res) >= B.proj_tol)) return fabs(res);
    const double disc = Bq * Bq - 4.0 * A * C;
    if (disc >= 0.0) {
        const double q = -0.5 * (Bq + copysign(sqrt(disc), Bq));
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
            if (fabs(x - ut) < dist) best = x;
        }
        y[3] = best;
    }
    return fabs(res);
}

// theta outside [0, pi]: the same point with theta reflected and phi + pi;
// the derivative f (when given) follows.
__device__ __forceinline__ void bl_reflect(double* y, double* f) {
    double th = y[1];
    if (th < 0.0) {
        th = -th;
    } else if (th > kPi) {
        th = 2.0 * kPi - th;
    } else {
        return;
    }
    y[1] = th;
    y[2] += kPi;
    y[5] = -y[5];
    if (f) {
        f[1] = -f[1];
        f[5] = -f[5];
    }
}

// E = -u_t, L = u_phi, Carter Q = u_theta^2 + cos^2 (L^2 / sin^2 - a^2 E^2).
__device__ __forceinline__ void bl_invariants(const BlDesc& B, const double* y, double& E, double& L, double& Q) {
    KnGeom G;
    kn_geometry<false>(B.m, B.a, B.q2, y[0], y[1], G);
    E = -(G.g[0] * y[3] + G.g[1] * y[6]);
    L = G.g[1] * y[3] + G.g[4] * y[6];
    const double pth = G.g[3] * y[5];
    Q = pth * pth + G.cos1 * G.cos1 * (L * L / G.sin2 - B.a * B.a * E * E);
}

// Pixel -> pinhole direction -> spherical components at the observer ->
// ZAMO light ray (software_compute_engine.hpp:3843-3862, 3912-3938, 1347-1350).
template <int BLOCK>
__device__ __noinline__ void bl_init_ray(const BlDesc* __restrict__ Bp, uint64_t local, BlCold<BLOCK>& S, int tid,
                                         double* __restrict__ y) {
    const BlDesc& B = *Bp;
    const uint32_t row = static_cast<uint32_t>(local / B.ncols);
    const uint32_t col = static_cast<uint32_t>(local - static_cast<uint64_t>(row) * B.ncols);
    const double px = static_cast<double>(B.col0 + col);
    const double py = static_cast<double>(B.row0 + row);
    const double v = 1.0 - (py + 0.5) / static_cast<double>(B.height) * 2.0;
    const double u = ((px + 0.5) / static_cast<double>(B.width) * 2.0 - 1.0) * B.aspect;
    const double n2 = v * B.tan_half_fov, n3 = u * B.tan_half_fov;
    const double len = sqrt(1.0 + n2 * n2 + n3 * n3);
    const double inv = (len > 0.0) ? (1.0 / len) : 1.0;
    const double nl0 = inv, nl1 = n2 * inv, nl2 = n3 * inv;
    double d[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) d[i] = nl0 * B.fwd[i] + nl2 * B.rgt[i] + nl1 * B.up[i];
    const double st = B.st, ct = B.ct, sp = B.sp, cp = B.cp;
    const double n_r = d[0] * (st * cp) + d[1] * (st * sp) + d[2] * ct;
    const double n_th = d[0] * (ct * cp) + d[1] * (ct * sp) + d[2] * (-st);
    const double n_ph = d[0] * (-sp) + d[1] * cp;
    const double nlen = sqrt(n_r * n_r + n_th * n_th + n_ph * n_ph);
    const double ninv = (nlen > 0.0) ? 1.0 / nlen : 1.0;
    y[0] = B.r_obs;
    y[1] = B.th_obs;
    y[2] = B.ph_obs;
    y[3] = B.e0_t;
    y[4] = -n_r * ninv * B.e_r;
    y[5] = -n_th * ninv * B.e_th;
    y[6] = B.e0_phi - n_ph * ninv * B.e_ph;
    double E, L, Q;
    bl_invariants(B, y, E, L, Q);
    S.e0[tid] = E;
    S.l0[tid] = L;
    S.q0[tid] = Q;
    S.lambda[tid] = 0.0;
    S.dH[tid] = 0.0;
    S.local[tid] = local;
}

// Sky-lookup direction of a (reflected) Boyer-Lindquist state: the
// orthonormal-frame velocity (sqrt(g_rr) u^r, sqrt(g_thth) u^th, sqrt(g_phph)
// u^ph) mapped to a Cartesian direction of travel (software_compute_engine.hpp:
// 1581-1589, local_frame_to_travel_direction :1148-1168).
__device__ void bl_exit_direction(const BlDesc& B, const double* y, double* e) {
    const double r = y[0], st = sin(y[1]), ct = cos(y[1]), sp = sin(y[2]), cp = cos(y[2]);
    const double a2 = B.a * B.a, r2a2 = r * r + a2;
    const double sigma = r * r + a2 * ct * ct;
    const double delta = r * r - 2.0 * B.m * r + a2 + B.q2;
    const double g_rr = sigma / delta;
    const double g_pp = (r2a2 * r2a2 - a2 * delta * st * st) * st * st / sigma;
    const double lr = sqrt(fmax(g_rr, 0.0)) * y[4], lt = sqrt(fmax(sigma, 0.0)) * y[5], lp = sqrt(fmax(g_pp, 0.0)) * y[6];
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

// Continuation end of a Boyer-Lindquist ray at state yin (unreflected), with
// the sky-lookup direction there when the sky is on.
__device__ __noinline__ void bl_cont_finish(const ContOut& C, const BlDesc& B, uint64_t o, uint32_t n_cross,
                                            uint32_t status, const double* yin) {
    double e[3];
    const double* ep = nullptr;
    if (C.exit) {
        double y[NB];
        for (int i = 0; i < NB; ++i) y[i] = yin[i];
        bl_reflect(y, nullptr);
        bl_exit_direction(B, y, e);
        ep = e;
    }
    cont_finish(C, o, n_cross, status, yin[0], B.m, ep);
}

template <int BLOCK>
__device__ __noinline__ void bl_finish(const BlDesc* __restrict__ Bp, BlCold<BLOCK>& S, int tid, const double* yin,
                                       uint32_t status, uint32_t flags, uint32_t acc, uint32_t rej, double r_hit,
                                       double g, const OutPtrs& out) {
    const BlDesc& B = *Bp;
    double y[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) y[i] = yin[i];
    bl_reflect(y, nullptr);
    double E, L, Q;
    bl_invariants(B, y, E, L, Q);
    const double e0 = S.e0[tid];
    const uint64_t o = B.out_offset + S.local[tid];
    const rt_ray_out& R = out.rays;
    if (R.status) R.status[o] = status;
    if (R.flags) R.flags[o] = flags;
    if (R.steps_accepted) R.steps_accepted[o] = acc;
    if (R.steps_rejected) R.steps_rejected[o] = rej;
    if (R.r) R.r[o] = y[0];
    if (R.theta) R.theta[o] = y[1];
    if (R.phi) R.phi[o] = y[2];
    if (R.r_hit) R.r_hit[o] = r_hit;
    if (R.g) R.g[o] = g;
    if (R.lambda) R.lambda[o] = S.lambda[tid];
    if (R.dH) R.dH[o] = S.dH[tid];
    if (R.dE) R.dE[o] = E / e0 - 1.0;
    if (R.dLz) R.dLz[o] = (L - S.l0[tid]) / e0;
    if (R.dQ) R.dQ[o] = (Q - S.q0[tid]) / (e0 * e0);
    if (R.body) R.body[o] = (status == RT_RAY_DISK || status == RT_RAY_CAPTURED) ? 0u : RT_BODY_NONE;
    if (R.exit_x || R.exit_y || R.exit_z) {
        double e[3] = {NAN, NAN, NAN};
        if (status == RT_RAY_ESCAPED) bl_exit_direction(B, y, e);
        if (R.exit_x) R.exit_x[o] = e[0];
        if (R.exit_y) R.exit_y[o] = e[1];
        if (R.exit_z) R.exit_z[o] = e[2];
    }
    if (out.pixels) {
        const uint32_t pflags = (status == RT_RAY_CAPTURED)  ? RT_PIXEL_HORIZON_ABSORBED
                                : (status == RT_RAY_ESCAPED) ? RT_PIXEL_CELESTIAL_HIT
                                : (status == RT_RAY_DISK)    ? RT_PIXEL_ACCRETION_DISK_HIT
                                                             : 0u;
        float4* p4 = reinterpret_cast<float4*>(out.pixels + o);
        p4[0] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        reinterpret_cast<uint4*>(p4)[1] = make_uint4(__float_as_uint(static_cast<float>(g)),
                                                     __float_as_uint(static_cast<float>(-S.lambda[tid])), pflags, acc);
    }
}

// VOL: hydro model 2, each accepted step's chord through the Fishbone-Moncrief
// torus gathered into the ray's record (args.cont.vol)
template <int BLOCK, bool VOL = false>
__global__ void __launch_bounds__(BLOCK, 384 / BLOCK) bl_trace_kernel(BlArgs args) {
    __shared__ BlCold<BLOCK> S;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const unsigned lt_mask = (1u << lane) - 1u;

    double y[NB], k1[NB];
    double h = 0.0;
    float lnp = 0.0f;
    bool has_hist = false;
    int can_early = 0;  // -1: undecided (Carter test when first inside r_early)
    uint32_t acc = 0, rej = 0, flags = 0, bidx = 0, guard = 0;
    uint32_t n_cross = 0;  // disk crossings so far (translucent-disk continuation)
    int mode = BL_IDLE;
#pragma unroll
    for (int i = 0; i < NB; ++i) y[i] = k1[i] = 0.0;
    bool queue_open = true;
    uint64_t chunk_next = 0, chunk_end = 0;
    uint32_t n_att = 0, n_acc = 0, n_rays = 0;

    for (;;) {
        // refill idle lanes from the warp's chunk, then from a new chunk (one atomic)
        const unsigned idle = __ballot_sync(FULL, mode == BL_IDLE);
        const int n_idle = __popc(idle);
        if ((queue_open || chunk_next < chunk_end) && n_idle > 0 &&
            (n_idle >= static_cast<int>(args.refill_threshold) || n_idle == 32)) {
            const uint64_t avail = chunk_end - chunk_next;
            uint64_t base2 = 0;
            bool got2 = false;
            if (avail < static_cast<uint64_t>(n_idle) && queue_open) {
                const int leader = __ffs(idle) - 1;
                unsigned long long b = 0;
                if (lane == leader) b = atomicAdd(args.queue, static_cast<unsigned long long>(args.claim));
                b = __shfl_sync(FULL, b, leader);
                if (b >= args.total_rays) {
                    queue_open = false;
                } else {
                    base2 = b;
                    got2 = true;
                    if (b + args.claim >= args.total_rays) queue_open = false;
                }
            }
            const uint64_t used_old = (avail < static_cast<uint64_t>(n_idle)) ? avail : n_idle;
            if (mode == BL_IDLE) {
                const uint64_t rank = static_cast<uint64_t>(__popc(idle & lt_mask));
                uint64_t rid = ~0ull;
                if (rank < avail) rid = chunk_next + rank;
                else if (got2) rid = base2 + (rank - avail);
                if (rid < args.total_rays) {
                    uint32_t lo = 0, hi = args.n_bundles;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (args.bundles[mid].ray_begin <= rid) lo = mid; else hi = mid;
                    }
                    bidx = lo;
                    const BlDesc* Bp = args.bundles + lo;
                    bl_init_ray<BLOCK>(Bp, rid - Bp->ray_begin, S, tid, y);
                    bl_rhs(Bp->m, Bp->a, Bp->q2, y, k1);
                    h = -Bp->h0;
                    lnp = 0.0f;
                    has_hist = false;
                    can_early = (Bp->flags & BF_EARLY_CAPTURE) ? -1 : 0;
                    n_cross = 0;
                    acc = rej = flags = guard = 0;
                    mode = BL_STEP;
                    ++n_rays;
                }
            }
            if (got2) {
                chunk_next = base2 + (static_cast<uint64_t>(n_idle) - used_old);
                chunk_end = base2 + args.claim;
                if (chunk_end > args.total_rays) chunk_end = args.total_rays;
            } else {
                chunk_next += used_old;
            }
        }
        if (__ballot_sync(FULL, mode != BL_IDLE) == 0) {
            if (!queue_open && chunk_next >= chunk_end) break;
            continue;
        }
        if (mode == BL_IDLE) continue;

        const BlDesc* Bp = args.bundles + bidx;
        const BlDesc& B = *Bp;
        // termination before the attempt; a backstop on loop iterations per ray
        uint32_t term = 0;
        if (++guard > B.max_steps + 64u) {
            flags |= RT_RAYFLAG_MAX_STEPS;
            term = RT_RAY_UNFINISHED + 16;
        } else if (y[0] < B.r_capture) {
            term = RT_RAY_CAPTURED;
        } else if (y[0] > B.r_esc) {
            term = RT_RAY_ESCAPED;
        } else if (acc + rej >= B.max_steps) {
            flags |= RT_RAYFLAG_MAX_STEPS;
            term = RT_RAY_UNFINISHED + 16;
        } else {
            const double cap = B.cap_c * fmax(y[0] - B.rh, 0.01 * B.m);
            if (fabs(h) > cap) h = -cap;
            if (fabs(h) < 1e-8) {
                flags |= RT_RAYFLAG_STEP_UNDERFLOW;
                term = RT_RAY_CAPTURED;
            }
        }
        if (term) {
            if (n_cross == 0) bl_finish<BLOCK>(Bp, S, tid, y, term & 15u, flags, acc, rej, NAN, 1.0, args.out);
            if (args.cont.cross) bl_cont_finish(args.cont, B, B.out_offset + S.local[tid], n_cross, term & 15u, y);
            mode = BL_IDLE;
            continue;
        }

        const double hh = h;
        double y5[NB];
        double err = bl_stages<BLOCK>(B, y, k1, hh, S, tid, y5);
        if (!(err <= 1e300)) err = 1e300;
        ++n_att;
        if (err > 1.0) {
            ++rej;
            const float le = __log2f(fmaxf(static_cast<float>(err), 1e-12f));
            const float factor = pi30_factor(le, has_hist ? lnp : le, 4.0f);
            lnp = le;
            has_hist = true;
            h = -fabs(h) * clampd(0.9 * static_cast<double>(factor), 0.1, 0.9);
            continue;
        }
        ++acc;
        ++n_acc;
        double k7[NB];
#pragma unroll
        for (int i = 0; i < NB; ++i) k7[i] = S.k[5][i][tid];
        bool finite = true;
#pragma unroll
        for (int i = 0; i < NB; ++i) finite = finite && isfinite(y5[i]);
        if (!finite) {
            if (n_cross == 0)
                bl_finish<BLOCK>(Bp, S, tid, y, RT_RAY_CAPTURED, flags | RT_RAYFLAG_NONFINITE, acc, rej, NAN, 1.0,
                                 args.out);
            if (args.cont.cross)
                bl_cont_finish(args.cont, B, B.out_offset + S.local[tid], n_cross, RT_RAY_CAPTURED, y);
            mode = BL_IDLE;
            continue;
        }
        // disk: the theta = pi/2 crossing of this step, when its root lies on the disk
        if (B.flags & BF_DISK) {
            const double f0 = y[1] - kHalfPi, f1 = y5[1] - kHalfPi;
            if (f0 * f1 <= 0.0 && f0 != f1) {
                const double sl = f0 / (f0 - f1);
                const double re = y[0] + sl * (y5[0] - y[0]);
                const double margin = 0.05 * re + 0.5 * B.m;
                if (re >= B.r_in - margin && re <= B.r_out + margin) {
                    double co[4][NB];
                    bl_dense_coeffs<BLOCK>(y, y5, k1, k7, hh, S, tid, co);
                    const double t = bl_dense_root(y, co, 1, kHalfPi, f0, f1, 1e-15);
                    double yr[NB];
#pragma unroll
                    for (int i = 0; i < NB; ++i) yr[i] = bl_dense_at(y, co, i, t);
                    const double rr = yr[0];
                    if (rr >= B.r_in && rr <= B.r_out && rr > B.rh * 1.02) {
                        double E, L, Q;
                        bl_invariants(B, yr, E, L, Q);
                        const double g = disk_redshift(B.m, B.a, rr, L / E);
                        if (n_cross == 0) {
                            // lambda at the root, one rounding with or without the continuation
                            const double lambda_step = S.lambda[tid];
                            S.lambda[tid] = fma(t, hh, lambda_step);
                            bl_finish<BLOCK>(Bp, S, tid, yr, RT_RAY_DISK, flags, acc, rej, rr, g, args.out);
                            S.lambda[tid] = lambda_step;
                        }
                        mode = BL_IDLE;
                        if (!args.cont.cross) continue;
                        // translucent disk: record the crossing (at the record's azimuth,
                        // that of the reflected root point) and go on through it
                        double yp[NB];
#pragma unroll
                        for (int i = 0; i < NB; ++i) yp[i] = yr[i];
                        bl_reflect(yp, nullptr);
                        const uint64_t o = B.out_offset + S.local[tid];
                        cont_record(args.cont, o, n_cross, rr, yp[2], g);
                        ++n_cross;
                        if (n_cross >= kMaxCrossings) {
                            bl_cont_finish(args.cont, B, o, n_cross, RT_RAY_UNFINISHED, yr);
                            continue;
                        }
                        mode = BL_STEP;
                    }
                }
            }
        }
        // capture / escape / certain capture inside this step: the terminal point on
        // the dense output at the threshold radius
        {
            double target = 0.0;
            uint32_t tterm = 0;
            const double rn = y5[0];
            if (rn < B.r_capture) {
                tterm = RT_RAY_CAPTURED;
                target = B.r_capture;
            } else if (rn > B.r_esc) {
                tterm = RT_RAY_ESCAPED;
                target = B.r_esc;
            } else if (can_early != 0 && rn < B.r_early) {
                if (can_early < 0) {
                    const double e0 = S.e0[tid];
                    can_early = shadow_distance(B.m, B.a, B.q2, B.rh, S.l0[tid] / e0, S.q0[tid] / (e0 * e0)) >
                                kEarlyCaptureMargin;
                }
                // u^r > 0 with h < 0: r decreases along the trace
                if (can_early > 0 && y5[4] > 0.0) {
                    tterm = RT_RAY_CAPTURED;
                    flags |= RT_RAYFLAG_EARLY_CAPTURE;
                    target = B.r_early;
                }
            }
            if (tterm) {
                double yt[NB];
                const double f0 = y[0] - target, f1 = rn - target;
                if ((f0 > 0.0) != (f1 > 0.0)) {
                    double co[4][NB];
                    bl_dense_coeffs<BLOCK>(y, y5, k1, k7, hh, S, tid, co);
                    const double t = bl_dense_root(y, co, 0, target, f0, f1, 1e-13 * target);
#pragma unroll
                    for (int i = 0; i < NB; ++i) yt[i] = bl_dense_at(y, co, i, t);
                    S.lambda[tid] += t * hh;
                } else {
#pragma unroll
                    for (int i = 0; i < NB; ++i) yt[i] = y5[i];
                    S.lambda[tid] += hh;
                }
                if (n_cross == 0) bl_finish<BLOCK>(Bp, S, tid, yt, tterm, flags, acc, rej, NAN, 1.0, args.out);
                if (args.cont.cross) bl_cont_finish(args.cont, B, B.out_offset + S.local[tid], n_cross, tterm, yt);
                mode = BL_IDLE;
                continue;
            }
        }
        S.dH[tid] = fmax(S.dH[tid], bl_project(B, y5));
        bl_reflect(y5, k7);
        if constexpr (VOL) {
            // the step's chord through the torus, L / E taken as u^phi r^2 sin^2 theta
            // at the step's end (software_compute_engine.hpp:1529-1537)
            const double s0 = sin(y[1]), s1 = sin(y5[1]);
            const double from[3] = {y[0] * s0 * cos(y[2]), y[0] * s0 * sin(y[2]), y[0] * cos(y[1])};
            const double to[3] = {y5[0] * s1 * cos(y5[2]), y5[0] * s1 * sin(y5[2]), y5[0] * cos(y5[1])};
            fm_segment(*args.cont.shade, from, to, y5[6] * (y5[0] * y5[0] * s1 * s1),
                       args.cont.vol + (B.out_offset + S.local[tid]) * VL_COUNT);
        }
        S.lambda[tid] += hh;
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            y[i] = y5[i];
            k1[i] = k7[i];
        }
        float factor = 5.0f;
        if (err != 0.0) {
            const float le = __log2f(fmaxf(static_cast<float>(err), 1e-12f));
            factor = pi30_factor(le, has_hist ? lnp : le, 5.0f);
            lnp = le;
            has_hist = true;
        }
        h = -clampd(fabs(h) * clampd(0.9 * static_cast<double>(factor), 0.2, 5.0), 1e-8, 1e13);
    }

    unsigned long long a64 = n_att, c64 = n_acc, r64 = n_rays;
    for (int off = 16; off > 0; off >>= 1) {
        a64 += __shfl_down_sync(FULL, a64, off);
        c64 += __shfl_down_sync(FULL, c64, off);
        r64 += __shfl_down_sync(FULL, r64, off);
    }
    if (lane == 0) {
        atomicAdd(args.stats + ST_RAYS, r64);
        atomicAdd(args.stats + ST_ATTEMPTS, a64);
        atomicAdd(args.stats + ST_ACCEPTED, c64);
        atomicAdd(args.stats + ST_FP64_ATTEMPTS, a64);
    }
}

template __global__ void bl_trace_kernel<128, false>(BlArgs);
template __global__ void bl_trace_kernel<128, true>(BlArgs);

}  // namespace

uint32_t bl_trace_grid(int sm_count) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bl_trace_kernel<128, false>, 128, 0) != cudaSuccess) {
        cudaGetLastError();
        occ = 1;
    }
    return static_cast<uint32_t>(sm_count) * static_cast<uint32_t>(occ > 1 ? occ : 1);
}

void launch_bl_trace(const BlArgs& args, uint32_t grid, void* stream) {
    if (args.cont.vol)
        bl_trace_kernel<128, true><<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(args);
    else
        bl_trace_kernel<128, false><<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(args);
}

}  // namespace relsim
