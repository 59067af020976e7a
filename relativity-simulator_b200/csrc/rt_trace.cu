// rt_trace.cu -- persistent backward null-geodesic tracer for sm_100a.
//
// One ray per lane, state in registers.  Warps claim rays from a global work
// counter; when at least `refill_threshold` lanes of a warp are idle the warp
// claims that many consecutive rays with one atomic (ballot + popc rank), so
// lanes whose rays terminated early are refilled instead of idling while the
// warp's longest ray finishes.
//
// Per ray: Dormand-Prince 5(4) on the Kerr-Schild Hamiltonian state
// (x, p) with p_t = -1 (kerr_schild_null_integrator.hpp:72-114), PI30 control
// (step_controller.hpp:51-58, accept/reject scaling rk45_adaptive.hpp:294-310),
// FSAL reuse of the last stage, a step cap |h| <= c max(r - r_+, 0.01 M),
// projection onto H = 0 after each accepted step, and classification:
// captured (r < capture_scale r_+, software_compute_engine.hpp:1667-1671),
// escaped (r > escape radius, :1672-1675), disk (first z = 0 crossing on
// [r_in, r_out], root by Illinois regula falsi on the step fraction), with the
// Carter certain-capture early-out (carter_ray_classifier.hpp:146-150).
//
// The disk root solve reuses the main stage code: a lane in ROOT mode runs
// its next DP5 evaluation at a fraction of the step instead of a full step, so
// all lanes of a warp share one instruction stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "rt_device.cuh"
#include "rt_internal.h"

namespace relsim {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kEarlyCaptureMargin = 1e-4;  // M, distance to the critical curve

enum LaneMode : int { MODE_IDLE = 0, MODE_STEP = 1, MODE_ROOT = 2, MODE_REDO = 3 };

struct RayLane {
    double y[6];
    double k1[6];
    double r;        // BL radius of y
    double h;        // next step (negative)
    double ln_prev;  // log of the previous error (PI30 history)
    double lambda;
    double dH;
    double lz0, q0;
    // root solve
    double lo, hi, flo, fhi, troot;
    uint64_t local;  // ray index inside its bundle
    uint32_t bidx;
    uint32_t acc, rej, flags;
    int mode;
    int side, rit;
    int wind;
    float raw_prev;
    bool has_hist;
    bool can_early;
};

__device__ __forceinline__ double clampd(double v, double lo, double hi) { return fmin(fmax(v, lo), hi); }

// Signed distance of (xi, eta) from the Kerr critical curve in impact
// parameter (units of M): the smallest local minimum R_min of the radial
// quartic R(r) = r^4 + P r^2 + Qc r - a^2 eta (carter_ray_classifier.hpp:132-135)
// outside r_+ is moved to zero by d_eta = R_min / Delta.  > 0: no turning point.
__device__ double shadow_distance(double M, double a, double rh, double xi, double eta) {
    const double a2 = a * a;
    const double P = a2 - xi * xi - eta;
    const double Qc = 2.0 * M * (eta + (xi - a) * (xi - a));
    const double R0 = -a2 * eta;
    const double pp = 0.5 * P, qq = 0.25 * Qc;
    double roots[3];
    int n = 0;
    const double disc = -(4.0 * pp * pp * pp + 27.0 * qq * qq);
    if (disc > 0.0 && pp < 0.0) {
        const double m2 = 2.0 * sqrt(-pp / 3.0);
        const double arg = clampd(3.0 * qq / (pp * m2), -1.0, 1.0);
        const double th = acos(arg) / 3.0;
        for (int k = 0; k < 3; ++k) roots[n++] = m2 * cos(th - 2.0 * kPi * k / 3.0);
    } else {
        const double sq = sqrt(fmax(qq * qq / 4.0 + pp * pp * pp / 27.0, 0.0));
        roots[n++] = cbrt(-qq / 2.0 + sq) + cbrt(-qq / 2.0 - sq);
    }
    double best = INFINITY, best_r = 0.0;
    for (int i = 0; i < n; ++i) {
        const double r = roots[i];
        if (!(r > rh)) continue;
        if (12.0 * r * r + 2.0 * P <= 0.0) continue;
        const double R = ((r * r + P) * r + Qc) * r + R0;
        if (R < best) {
            best = R;
            best_r = r;
        }
    }
    if (!isfinite(best)) return INFINITY;
    const double delta = best_r * best_r - 2.0 * M * best_r + a2;
    const double b = sqrt(fmax(eta + xi * xi, 1e-30));
    return best / fmax(delta, 1e-30) / (2.0 * b);
}

// Carter constant with E = 1, mu = 0 (kerr_invariants.hpp:45-48); BL p_theta
// from the Kerr-Schild covector through dx^i/dtheta of the map at
// kerr_schild_null_integrator.hpp:47-53.
__device__ double carter_q(const double* y, double a) {
    const double r = sqrt(bl_r2<double>(y[0], y[1], y[2], a * a));
    const double cos_t = clampd(y[2] / r, -1.0, 1.0);
    const double sin2 = fmax((y[0] * y[0] + y[1] * y[1]) / (r * r + a * a), 1e-30);
    const double sin_t = sqrt(sin2);
    const double p_theta = (y[0] * y[3] + y[1] * y[4]) * cos_t / sin_t - r * sin_t * y[5];
    const double lz = y[0] * y[4] - y[1] * y[3];
    return p_theta * p_theta + cos_t * cos_t * (-a * a + lz * lz / sin2);
}

__device__ __forceinline__ float raw_phi32(const double* y, double a, double r) {
    return atan2f(static_cast<float>(y[1]), static_cast<float>(y[0])) -
           atan2f(static_cast<float>(a), static_cast<float>(r));
}

// Ray generation (software_compute_engine.hpp:3843-3862, :3932-3938, :1637-1650,
// camera_projections.hpp:27-40) and the initial null covector
// (kerr_schild_null_integrator.hpp:179-193) from the bundle's precomputed tetrad.
__device__ void init_ray(const BundleDesc& B, uint64_t local, RayLane& L) {
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
    const double ow[3] = {n_r * st * cp + n_th * ct * cp - n_ph * sp, n_r * st * sp + n_th * ct * sp + n_ph * cp,
                          n_r * ct - n_th * st};
    double v4[4] = {B.u0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) v4[c] -= ow[i] * B.e[i][c];
    const double lv = v4[0] + B.kf[0] * v4[1] + B.kf[1] * v4[2] + B.kf[2] * v4[3];
    const double p_t = -v4[0] + B.two_h * lv;
    const double inv_e = 1.0 / fmax(-p_t, 1e-12);
    L.y[0] = B.x0[0];
    L.y[1] = B.x0[1];
    L.y[2] = B.x0[2];
    L.y[3] = (v4[1] + B.two_h * lv * B.kf[0]) * inv_e;
    L.y[4] = (v4[2] + B.two_h * lv * B.kf[1]) * inv_e;
    L.y[5] = (v4[3] + B.two_h * lv * B.kf[2]) * inv_e;
    L.lz0 = L.y[0] * L.y[4] - L.y[1] * L.y[3];
    L.q0 = carter_q(L.y, B.a);
    L.can_early = (B.flags & BF_EARLY_CAPTURE) && shadow_distance(B.m, B.a, B.rh, L.lz0, L.q0) > kEarlyCaptureMargin;
    double hf, s;
    L.r = ks_rhs<double>(L.y, B.m, B.a, L.k1, hf, s);
    L.h = -B.h0;
    L.ln_prev = 0.0;
    L.has_hist = false;
    L.lambda = 0.0;
    L.dH = 0.0;
    L.acc = L.rej = L.flags = 0;
    L.wind = B.wind0;
    L.raw_prev = static_cast<float>(B.raw_phi0);
    L.local = local;
}

// Disk redshift of a circular orbit (accretion_disk_model.hpp:205-225).
__device__ double disk_redshift(double M, double a, double r, double lz) {
    const double am = fabs(a);
    const double sm = sqrt(fmax(M, 1e-12));
    const double sr = sqrt(fmax(r, 1e-12));
    const double r15 = r * sr;
    const double ang = sm / (r15 + am * sm);
    const double bracket = fmax(r15 - 3.0 * M * sr + 2.0 * am * sm, 1e-9);
    const double omega = (a < 0.0) ? -ang : ang;
    const double ut = (r15 + am * sm) / (sqrt(r15) * sqrt(bracket));
    const double den = ut * (1.0 - omega * lz);
    return (fabs(den) > 1e-9) ? clampd(1.0 / den, 0.05, 4.0) : 1.0;
}

// Write the ray's record and pixel, then free the lane.
__device__ void finish_ray(const BundleDesc& B, RayLane& L, uint32_t status, double r_hit, double g,
                           const OutPtrs& out) {
    const double a = B.a;
    const double* y = L.y;
    const double r = sqrt(bl_r2<double>(y[0], y[1], y[2], a * a));
    const double rho = sqrt(fmax(r * r - y[2] * y[2], 0.0));
    const double theta = atan2(rho, y[2]);
    const double raw = atan2(y[1], y[0]) - atan2(a, r);
    // last winding update against the tracked azimuth (kerr_schild_null_integrator.hpp:61-63)
    const float raw32 = static_cast<float>(raw);
    const float dr = raw32 - L.raw_prev;
    int wind = L.wind;
    if (dr > static_cast<float>(kPi)) wind -= 1;
    if (dr < -static_cast<float>(kPi)) wind += 1;
    const double phi = raw + kTwoPi * static_cast<double>(wind);
    // invariants at the end
    double kf[3], hf;
    ks_field64(y, B.m, a, kf, hf);
    const double kp = kf[0] * y[3] + kf[1] * y[4] + kf[2] * y[5];
    const double pp = y[3] * y[3] + y[4] * y[4] + y[5] * y[5];
    const double qa = 1.0 + 2.0 * hf, qb = 2.0 * hf * kp, qc = pp - 2.0 * hf * kp * kp;
    const double energy = (-qb + sqrt(fmax(qb * qb + qa * qc, 0.0))) / qa;
    const double lz = y[0] * y[4] - y[1] * y[3];
    const double q = carter_q(y, a);

    const uint64_t o = B.out_offset + L.local;
    const rt_ray_out& R = out.rays;
    if (R.status) R.status[o] = status;
    if (R.flags) R.flags[o] = L.flags;
    if (R.steps_accepted) R.steps_accepted[o] = L.acc;
    if (R.steps_rejected) R.steps_rejected[o] = L.rej;
    if (R.r) R.r[o] = r;
    if (R.theta) R.theta[o] = theta;
    if (R.phi) R.phi[o] = phi;
    if (R.r_hit) R.r_hit[o] = r_hit;
    if (R.g) R.g[o] = g;
    if (R.lambda) R.lambda[o] = L.lambda;
    if (R.dH) R.dH[o] = L.dH;
    if (R.dE) R.dE[o] = energy - 1.0;
    if (R.dLz) R.dLz[o] = lz - L.lz0;
    if (R.dQ) R.dQ[o] = q - L.q0;
    if (out.pixels) {
        rt_pixel_out px;
        px.r = px.g = px.b = 0.0f;
        px.a = 1.0f;
        px.redshift = static_cast<float>(g);
        px.affine_parameter = static_cast<float>(-L.lambda);
        px.status_flags = (status == RT_RAY_CAPTURED)  ? RT_PIXEL_HORIZON_ABSORBED
                          : (status == RT_RAY_ESCAPED) ? RT_PIXEL_CELESTIAL_HIT
                          : (status == RT_RAY_DISK)    ? RT_PIXEL_ACCRETION_DISK_HIT
                                                       : 0u;
        px.iterations_used = L.acc;
        reinterpret_cast<float4*>(out.pixels + o)[0] = make_float4(px.r, px.g, px.b, px.a);
        reinterpret_cast<uint4*>(out.pixels + o)[1] =
            make_uint4(__float_as_uint(px.redshift), __float_as_uint(px.affine_parameter), px.status_flags,
                       px.iterations_used);
    }
    L.mode = MODE_IDLE;
}

// Cubic Hermite interpolant of a step from its end points and FSAL slopes.
__device__ __forceinline__ void hermite(const double* y0, const double* f0, const double* y1, const double* f1,
                                        double h, double t, int n, double* out) {
    const double t2 = t * t, t3 = t2 * t;
    const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + t;
    const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
    for (int i = 0; i < n; ++i) out[i] = h00 * y0[i] + h10 * h * f0[i] + h01 * y1[i] + h11 * h * f1[i];
}

// Fraction of the step where the interpolated r_BL crosses `target`
// (Illinois regula falsi; returns 1 when the end points do not bracket it).
__device__ double crossing_fraction(const double* y0, const double* f0, const double* y1, const double* f1, double h,
                                    double a, double target) {
    const double a2 = a * a;
    double lo = 0.0, hi = 1.0;
    double flo = sqrt(bl_r2<double>(y0[0], y0[1], y0[2], a2)) - target;
    double fhi = sqrt(bl_r2<double>(y1[0], y1[1], y1[2], a2)) - target;
    if (!((flo > 0.0) != (fhi > 0.0))) return 1.0;
    int side = 0;
    double t = 1.0, x[3];
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        hermite(y0, f0, y1, f1, h, t, 3, x);
        const double ft = sqrt(bl_r2<double>(x[0], x[1], x[2], a2)) - target;
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

// Stages 2..6 and the 5th-order solution of a step hh from (y, k1)
// (rk45_adaptive.hpp:210-251).
__device__ __forceinline__ void dp5_stages(const double* y, const double* k1, double hh, double M, double a,
                                           double (&k)[6][6], double* y5) {
    double s[6], hf, sv;
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = y[i] + hh * (DP::A21 * k1[i]);
    ks_rhs<double>(s, M, a, k[1], hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = y[i] + hh * (DP::A31 * k1[i] + DP::A32 * k[1][i]);
    ks_rhs<double>(s, M, a, k[2], hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = y[i] + hh * (DP::A41 * k1[i] + DP::A42 * k[1][i] + DP::A43 * k[2][i]);
    ks_rhs<double>(s, M, a, k[3], hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i)
        s[i] = y[i] + hh * (DP::A51 * k1[i] + DP::A52 * k[1][i] + DP::A53 * k[2][i] + DP::A54 * k[3][i]);
    ks_rhs<double>(s, M, a, k[4], hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i)
        s[i] = y[i] + hh * (DP::A61 * k1[i] + DP::A62 * k[1][i] + DP::A63 * k[2][i] + DP::A64 * k[3][i] +
                            DP::A65 * k[4][i]);
    ks_rhs<double>(s, M, a, k[5], hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i)
        y5[i] = y[i] + hh * (DP::B1 * k1[i] + DP::B3 * k[2][i] + DP::B4 * k[3][i] + DP::B5 * k[4][i] +
                             DP::B6 * k[5][i]);
}

}  // namespace

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) trace_fp64_kernel_t(TraceArgs args) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;

    RayLane L;
    L.mode = MODE_IDLE;
    L.bidx = 0;
    bool queue_open = true;
    unsigned long long n_att = 0, n_acc = 0, n_rays = 0, n_rhs = 0;

    for (;;) {
        // ---- refill idle lanes from the global queue ----
        const unsigned idle = __ballot_sync(FULL, L.mode == MODE_IDLE);
        const int n_idle = __popc(idle);
        if (queue_open && n_idle > 0 && (n_idle >= static_cast<int>(args.refill_threshold) || n_idle == 32)) {
            const int leader = __ffs(idle) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(args.queue, static_cast<unsigned long long>(n_idle));
            base = __shfl_sync(FULL, base, leader);
            if (base + static_cast<unsigned long long>(n_idle) >= args.total_rays) queue_open = false;
            if (L.mode == MODE_IDLE) {
                const uint64_t rid = base + static_cast<uint64_t>(__popc(idle & lt_mask));
                if (rid < args.total_rays) {
                    // bundle of this ray: last bundle whose ray_begin <= rid
                    uint32_t lo = 0, hi = args.n_bundles;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (args.bundles[mid].ray_begin <= rid) lo = mid; else hi = mid;
                    }
                    L.bidx = lo;
                    init_ray(args.bundles[lo], rid - args.bundles[lo].ray_begin, L);
                    L.mode = MODE_STEP;
                    ++n_rays;
                    ++n_rhs;
                }
            }
        }
        if (__ballot_sync(FULL, L.mode != MODE_IDLE) == 0) {
            if (!queue_open) break;
            continue;
        }
        if (L.mode == MODE_IDLE) continue;

        const BundleDesc& B = args.bundles[L.bidx];
        const double M = B.m, a = B.a;
        double hh = L.h;
        bool attempt = true;
        if (L.mode == MODE_STEP) {
            // termination tests at the current point (software_compute_engine.hpp:1667-1675)
            if (L.r < B.r_capture) {
                finish_ray(B, L, RT_RAY_CAPTURED, NAN, 1.0, args.out);
                attempt = false;
            } else if (L.r > B.r_esc) {
                finish_ray(B, L, RT_RAY_ESCAPED, NAN, 1.0, args.out);
                attempt = false;
            } else if (L.acc + L.rej >= B.max_steps) {
                L.flags |= RT_RAYFLAG_MAX_STEPS;
                finish_ray(B, L, RT_RAY_UNFINISHED, NAN, 1.0, args.out);
                attempt = false;
            } else {
                const double cap = B.cap_c * fmax(L.r - B.rh, 0.01 * M);
                if (fabs(L.h) > cap) L.h = -cap;
                hh = L.h;
                if (fabs(hh) < 1e-8) {
                    L.flags |= RT_RAYFLAG_STEP_UNDERFLOW;
                    finish_ray(B, L, RT_RAY_CAPTURED, NAN, 1.0, args.out);
                    attempt = false;
                }
            }
        } else if (L.mode == MODE_ROOT) {
            double t = (L.lo * L.fhi - L.hi * L.flo) / (L.fhi - L.flo);
            if (!(t > L.lo && t < L.hi)) t = 0.5 * (L.lo + L.hi);
            L.troot = t;
            hh = t * L.h;
        }
        if (!attempt) continue;

        double k[6][6];
        double y5[6];
        dp5_stages(L.y, L.k1, hh, M, a, k, y5);
        n_rhs += 5;

        if (L.mode == MODE_ROOT) {
            const double ft = y5[2];
            ++L.rit;
            const bool done = (ft == 0.0) || (fabs(L.hi - L.lo) < 1e-15) ||
                              (fabs(ft) < 1e-13 * (1.0 + fabs(y5[0]) + fabs(y5[1]))) || (L.rit >= 60);
            if (done) {
                const double rr = sqrt(bl_r2<double>(y5[0], y5[1], y5[2], a * a));
                if (rr >= B.r_in && rr <= B.r_out && rr > B.rh * 1.02) {
                    L.lambda += L.troot * L.h;
                    for (int i = 0; i < 6; ++i) L.y[i] = y5[i];
                    finish_ray(B, L, RT_RAY_DISK, rr, disk_redshift(M, a, rr, L.lz0), args.out);
                } else {
                    L.mode = MODE_REDO;  // not on the disk: take the full step again
                }
            } else if ((ft > 0.0) == (L.fhi > 0.0)) {
                L.hi = L.troot;
                L.fhi = ft;
                if (L.side == -1) L.flo *= 0.5;
                L.side = -1;
            } else {
                L.lo = L.troot;
                L.flo = ft;
                if (L.side == 1) L.fhi *= 0.5;
                L.side = 1;
            }
            continue;
        }

        // full step: last stage (FSAL) and the error norm (rk45_adaptive.hpp:252-261)
        double hf5, s5;
        const double r5 = ks_rhs<double>(y5, M, a, k[0], hf5, s5);  // k[0] now holds k7
        n_rhs += 1;
        double err;
        {
            double num = 0.0, den = 1.0;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const double est = fabs(hh) * fabs(DP::E1 * L.k1[i] + DP::E3 * k[2][i] + DP::E4 * k[3][i] +
                                                   DP::E5 * k[4][i] + DP::E6 * k[5][i] + DP::E7 * k[0][i]);
                const double sc = B.rtol * fmax(fabs(L.y[i]), fabs(y5[i])) + B.atol;
                if (est * den > num * sc) {
                    num = est;
                    den = sc;
                }
            }
            err = num / den;
        }
        if (!(err <= 1e300)) err = 1e300;  // non-finite trial: reject with the largest cut

        if (L.mode == MODE_STEP) {
            ++n_att;
            if (err > 1.0) {
                // reject (rk45_adaptive.hpp:303-311)
                ++L.rej;
                const double le = log(fmax(err, 1e-12));
                const double lp = L.has_hist ? L.ln_prev : le;
                const double factor = exp(-(0.7 / 4.0) * le + (0.3 / 4.0) * (lp - le));
                L.ln_prev = le;
                L.has_hist = true;
                L.h = -fabs(L.h) * clampd(0.9 * factor, 0.1, 0.9);
                continue;
            }
            ++L.acc;
            ++n_acc;
            bool finite = true;
#pragma unroll
            for (int i = 0; i < 6; ++i) finite = finite && isfinite(y5[i]);
            if (!finite) {
                L.flags |= RT_RAYFLAG_NONFINITE;
                finish_ray(B, L, RT_RAY_CAPTURED, NAN, 1.0, args.out);
                continue;
            }
            if ((B.flags & BF_DISK) && L.y[2] * y5[2] <= 0.0 && L.y[2] != y5[2]) {
                const double sl = L.y[2] / (L.y[2] - y5[2]);
                const double xe = L.y[0] + sl * (y5[0] - L.y[0]);
                const double ye = L.y[1] + sl * (y5[1] - L.y[1]);
                const double re = sqrt(fmax(xe * xe + ye * ye - a * a, 0.0));
                const double margin = 0.05 * re + 0.5 * M;
                if (re >= B.r_in - margin && re <= B.r_out + margin) {
                    L.mode = MODE_ROOT;
                    L.lo = 0.0;
                    L.flo = L.y[2];
                    L.hi = 1.0;
                    L.fhi = y5[2];
                    L.side = 0;
                    L.rit = 0;
                    continue;
                }
            }
        }
        // accept, second half (also the REDO of a crossing off the disk)
        L.mode = MODE_STEP;
        {
            // capture / escape / certain capture inside this step: the terminal point is
            // interpolated to the threshold radius, independent of where the step ended
            double target = 0.0;
            uint32_t term = 0, tflag = 0;
            if (r5 < B.r_capture) {
                term = RT_RAY_CAPTURED;
                target = B.r_capture;
            } else if (r5 > B.r_esc) {
                term = RT_RAY_ESCAPED;
                target = B.r_esc;
            } else if (L.can_early && r5 < B.r_early) {
                // dr_BL/dlambda (kerr_invariants.hpp:140); the trace runs towards
                // decreasing lambda, so dr/dlambda > 0 means inwards
                const double r2 = r5 * r5, z = y5[2];
                const double drdl = (r2 * r5 * (y5[0] * k[0][0] + y5[1] * k[0][1]) + r5 * (r2 + a * a) * z * k[0][2]) /
                                    (r2 * r2 + a * a * z * z);
                if (drdl > 0.0) {
                    term = RT_RAY_CAPTURED;
                    tflag = RT_RAYFLAG_EARLY_CAPTURE;
                    target = B.r_early;
                }
            }
            if (term) {
                const double t = crossing_fraction(L.y, L.k1, y5, k[0], hh, a, target);
                double yt[6];
                hermite(L.y, L.k1, y5, k[0], hh, t, 6, yt);
#pragma unroll
                for (int i = 0; i < 6; ++i) L.y[i] = yt[i];
                L.lambda += t * hh;
                L.flags |= tflag;
                finish_ray(B, L, term, NAN, 1.0, args.out);
                continue;
            }
        }
        {
            // projection onto H = 0 (closest root, rk45_adaptive.hpp:126-134); n = dx/dl = k7[0..2],
            // k.n and |n|^2 from |k| = 1
            double* p = y5 + 3;
            const double pp = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
            const double res = 0.5 * (pp - 1.0 - 2.0 * hf5 * s5 * s5);
            L.dH = fmax(L.dH, fabs(res));
            if (fabs(res) >= B.proj_tol) {
                const double hs = hf5 * s5;
                const double kn = (s5 - 1.0) - 2.0 * hs;
                const double pn = pp - 2.0 * hs * (s5 - 1.0);
                const double nn = pp - 4.0 * hs * (s5 - 1.0) + 4.0 * hs * hs;
                const double qa = 0.5 * (nn - 2.0 * hf5 * kn * kn);
                const double qb = pn - 2.0 * hs * kn;
                const double disc = qb * qb - 4.0 * qa * res;
                if (disc >= 0.0) {
                    const double q = -0.5 * (qb + copysign(sqrt(disc), qb));
                    if (q != 0.0) {
                        const double alpha = res / q;
                        p[0] += alpha * k[0][0];
                        p[1] += alpha * k[0][1];
                        p[2] += alpha * k[0][2];
                    }
                }
            }
        }
        {
            const float raw = raw_phi32(y5, a, r5);
            const float d = raw - L.raw_prev;
            if (d > static_cast<float>(kPi)) L.wind -= 1;
            if (d < -static_cast<float>(kPi)) L.wind += 1;
            L.raw_prev = raw;
        }
        L.lambda += hh;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            L.y[i] = y5[i];
            L.k1[i] = k[0][i];
        }
        L.r = r5;
        double factor = 5.0;
        if (err != 0.0) {
            const double le = log(fmax(err, 1e-12));
            const double lp = L.has_hist ? L.ln_prev : le;
            factor = exp(-(0.7 / 5.0) * le + (0.3 / 5.0) * (lp - le));
            L.ln_prev = le;
            L.has_hist = true;
        }
        double ah = fabs(L.h) * clampd(0.9 * factor, 0.2, 5.0);
        L.h = -clampd(ah, 1e-8, 1e13);
    }

    // warp-reduced counters
    for (int off = 16; off > 0; off >>= 1) {
        n_att += __shfl_down_sync(FULL, n_att, off);
        n_acc += __shfl_down_sync(FULL, n_acc, off);
        n_rays += __shfl_down_sync(FULL, n_rays, off);
        n_rhs += __shfl_down_sync(FULL, n_rhs, off);
    }
    if (lane == 0) {
        atomicAdd(args.stats + ST_RAYS, n_rays);
        atomicAdd(args.stats + ST_ATTEMPTS, n_att);
        atomicAdd(args.stats + ST_ACCEPTED, n_acc);
        atomicAdd(args.stats + ST_RHS, n_rhs);
        atomicAdd(args.stats + ST_FP64_ATTEMPTS, n_att);
    }
}

template __global__ void trace_fp64_kernel_t<64>(TraceArgs);
template __global__ void trace_fp64_kernel_t<128>(TraceArgs);
template __global__ void trace_fp64_kernel_t<256>(TraceArgs);

namespace {
const void* kernel_for(uint32_t block, bool mixed) {
    (void)mixed;
    switch (block) {
        case 64: return reinterpret_cast<const void*>(&trace_fp64_kernel_t<64>);
        case 256: return reinterpret_cast<const void*>(&trace_fp64_kernel_t<256>);
        default: return reinterpret_cast<const void*>(&trace_fp64_kernel_t<128>);
    }
}
}  // namespace

int trace_occupancy(uint32_t block, bool mixed) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_for(block, mixed), static_cast<int>(block), 0) !=
        cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n;
}

void launch_trace(const TraceArgs& args, uint32_t grid, uint32_t block, bool mixed, cudaStream_t stream) {
    void* params[] = {const_cast<TraceArgs*>(&args)};
    cudaLaunchKernel(kernel_for(block, mixed), dim3(grid), dim3(block), params, 0, stream);
}

}  // namespace relsim
