// rt_ray.cuh -- per-ray pieces shared by the Kerr-Schild tracer kernels
// (rt_trace.cu: single kernel, far/near passes, finish pass): ray generation,
// termination records, the parked-ray format of the two-pass tracer, the
// dense-output disk root and the translucent-disk continuation.
//
// The cold per-lane state is passed as any structure with the SoA arrays
// lambda, dH, lz0, q0 and local, indexed by the caller's lane slot.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "rt_device.cuh"
#include "rt_internal.h"
#include "rt_shade.cuh"

namespace relsim {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kEarlyCaptureMargin = 1e-4;  // M, distance to the critical curve

enum LaneMode : int {
    MODE_IDLE = 0,
    MODE_STEP = 1,
    MODE_ROOT = 2,
    MODE_REDO = 3,
    MODE_PARK = 4,     // two-pass: to the other pass, state parked
    MODE_FINISHQ = 5,  // two-pass: a disk hit, root point parked for the finish pass
    MODE_CRITQ = 6     // far pass: a near-critical ray, to the critical pass (no state)
};

// Cold per-lane state, structure of arrays indexed by threadIdx.x.
template <int BLOCK>
struct Cold {
    double lambda[BLOCK];
    double dH[BLOCK];
    double lz0[BLOCK];
    double q0[BLOCK];
    double lo[BLOCK], hi[BLOCK], flo[BLOCK], fhi[BLOCK], troot[BLOCK];
    uint64_t local[BLOCK];
    int side[BLOCK], rit[BLOCK];
};

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

// Winding of atan2(y, x) across its branch cut between two points: the
// azimuth unwrapping of kerr_schild_null_integrator.hpp:61-63 counts a turn
// exactly when the segment crosses the negative x axis.
__device__ __forceinline__ int branch_winding(double x0, double y0, double x1, double y1) {
    if ((y0 < 0.0) == (y1 < 0.0)) return 0;
    const double xc = x0 + (x1 - x0) * (y0 / (y0 - y1));
    if (!(xc < 0.0)) return 0;
    return (y0 < 0.0) ? -1 : 1;
}

struct InitResult {
    double r;
    int can_early;  // -1: undecided; the Carter test runs when the ray first needs it
};

// Ray generation (software_compute_engine.hpp:3843-3862, :3932-3938, :1637-1650,
// camera_projections.hpp:27-40) and the initial null covector
// (kerr_schild_null_integrator.hpp:179-193) from the bundle's precomputed
// tetrad.  Writes y0 and k1 to xch[0..11] (a local array of the caller).
template <class ColdT>
__device__ __noinline__ InitResult init_ray(const BundleDesc* __restrict__ Bp, uint64_t local, ColdT& S,
                                            int tid, double* __restrict__ xch) {
    const BundleDesc& B = *Bp;
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
    double y[6], k1[6];
    y[0] = B.x0[0];
    y[1] = B.x0[1];
    y[2] = B.x0[2];
    y[3] = (v4[1] + B.two_h * lv * B.kf[0]) * inv_e;
    y[4] = (v4[2] + B.two_h * lv * B.kf[1]) * inv_e;
    y[5] = (v4[3] + B.two_h * lv * B.kf[2]) * inv_e;
    const double lz0 = y[0] * y[4] - y[1] * y[3];
    const double q0 = carter_q(y, B.a);
    double hf, s;
    InitResult res;
    res.r = ks_rhs<double>(y, B.m, B.a, k1, hf, s);
    res.can_early = (B.flags & BF_EARLY_CAPTURE) ? -1 : 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        xch[i] = y[i];
        xch[6 + i] = k1[i];
    }
    S.lz0[tid] = lz0;
    S.q0[tid] = q0;
    S.lambda[tid] = 0.0;
    S.dH[tid] = 0.0;
    S.local[tid] = local;
    return res;
}

// Terminal point, the ray's record and its pixel.  xch (a local array of the
// caller) holds the last accepted point in [0..5]; with interp_target > 0 it
// holds the step's y, k1, y5, k7 in [0..23] and the point is interpolated to
// r_BL = interp_target; for a disk hit the root state is in [12..17].
template <class ColdT>
__device__ __noinline__ void finish_ray(const BundleDesc* __restrict__ Bp, ColdT& S, int tid, uint32_t status,
                                        uint32_t flags, uint32_t acc, uint32_t rej, int wind, double interp_target,
                                        double hh, double r_hit, double g, const OutPtrs& out,
                                        const double* __restrict__ xch) {
    const BundleDesc& B = *Bp;
    const double a = B.a;
    double y[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] = xch[i];
    const double y_prev_x = y[0], y_prev_y = y[1];
    double lambda = S.lambda[tid];
    if (interp_target > 0.0) {
        double y0[6], f0[6], y1[6], f1[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            y0[i] = xch[i];
            f0[i] = xch[6 + i];
            y1[i] = xch[12 + i];
            f1[i] = xch[18 + i];
        }
        const double t = crossing_fraction(y0, f0, y1, f1, hh, a, interp_target);
        hermite(y0, f0, y1, f1, hh, t, 6, y);
        lambda += t * hh;
    } else if (status == RT_RAY_DISK) {
#pragma unroll
        for (int i = 0; i < 6; ++i) y[i] = xch[12 + i];
    }
    const double r = sqrt(bl_r2<double>(y[0], y[1], y[2], a * a));
    const double rho = sqrt(fmax(r * r - y[2] * y[2], 0.0));
    const double theta = atan2(rho, y[2]);
    wind += branch_winding(y_prev_x, y_prev_y, y[0], y[1]);
    const double phi = atan2(y[1], y[0]) - atan2(a, r) + kTwoPi * static_cast<double>(wind);
    // invariants at the end
    double kf[3], hf;
    ks_field64(y, B.m, a, kf, hf);
    const double kp = kf[0] * y[3] + kf[1] * y[4] + kf[2] * y[5];
    const double pp = y[3] * y[3] + y[4] * y[4] + y[5] * y[5];
    const double qa = 1.0 + 2.0 * hf, qb = 2.0 * hf * kp, qc = pp - 2.0 * hf * kp * kp;
    const double energy = (-qb + sqrt(fmax(qb * qb + qa * qc, 0.0))) / qa;
    const double lz = y[0] * y[4] - y[1] * y[3];
    const double q = carter_q(y, a);

    const uint64_t o = B.out_offset + S.local[tid];
    const rt_ray_out& R = out.rays;
    if (R.status) R.status[o] = status;
    if (R.flags) R.flags[o] = flags;
    if (R.steps_accepted) R.steps_accepted[o] = acc;
    if (R.steps_rejected) R.steps_rejected[o] = rej;
    if (R.r) R.r[o] = r;
    if (R.theta) R.theta[o] = theta;
    if (R.phi) R.phi[o] = phi;
    if (R.r_hit) R.r_hit[o] = r_hit;
    if (R.g) R.g[o] = g;
    if (R.lambda) R.lambda[o] = lambda;
    if (R.dH) R.dH[o] = S.dH[tid];
    if (R.dE) R.dE[o] = energy - 1.0;
    if (R.dLz) R.dLz[o] = lz - S.lz0[tid];
    if (R.dQ) R.dQ[o] = q - S.q0[tid];
    if (R.body) R.body[o] = (status == RT_RAY_DISK || status == RT_RAY_CAPTURED) ? 0u : RT_BODY_NONE;
    if (R.exit_x || R.exit_y || R.exit_z) {
        // sky-lookup direction of an escaped ray: -dx/dlambda at the terminal
        // state, normalised (software_compute_engine.hpp:1771-1775); each
        // component is written only where the caller asked for it
        double e[3] = {NAN, NAN, NAN};
        if (status == RT_RAY_ESCAPED) {
            const double sv = 1.0 + kp;
            const double v[3] = {y[3] - 2.0 * hf * sv * kf[0], y[4] - 2.0 * hf * sv * kf[1],
                                 y[5] - 2.0 * hf * sv * kf[2]};
            const double inv = 1.0 / fmax(sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), 1e-12);
#pragma unroll
            for (int i = 0; i < 3; ++i) e[i] = -v[i] * inv;
        }
        if (R.exit_x) R.exit_x[o] = e[0];
        if (R.exit_y) R.exit_y[o] = e[1];
        if (R.exit_z) R.exit_z[o] = e[2];
    }
    if (out.pixels) {
        // GpuPixelOutput (gpu_types.hpp:1111-1130); shading is not part of this path
        const uint32_t pflags = (status == RT_RAY_CAPTURED)  ? RT_PIXEL_HORIZON_ABSORBED
                                : (status == RT_RAY_ESCAPED) ? RT_PIXEL_CELESTIAL_HIT
                                : (status == RT_RAY_DISK)    ? RT_PIXEL_ACCRETION_DISK_HIT
                                                             : 0u;
        float4* p4 = reinterpret_cast<float4*>(out.pixels + o);
        p4[0] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        reinterpret_cast<uint4*>(p4)[1] = make_uint4(__float_as_uint(static_cast<float>(g)),
                                                     __float_as_uint(static_cast<float>(-lambda)), pflags, acc);
    }
}

// Resume a parked ray (two-pass tracer): its state from the park buffer, the
// cold per-lane state into shared memory, and the FSAL stage k1 = f(y) in FP64
// (one RHS per transition between passes).  Writes y, k1 to xch[0..11], h to
// xch[12], the parked words to uch[]; returns r_BL.
template <class ColdT>
__device__ __noinline__ double resume_ray(const BundleDesc* __restrict__ Bp, const ParkBuf pb, uint64_t ray,
                                          uint64_t local, ColdT& S, int tid, double* __restrict__ xch,
                                          uint32_t* __restrict__ uch) {
    const uint64_t n = pb.n;
    double y[6], k1[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] = pb.d[(PD_Y + i) * n + ray];
    xch[12] = pb.d[PD_H * n + ray];
    S.lambda[tid] = pb.d[PD_LAMBDA * n + ray];
    S.dH[tid] = pb.d[PD_DH * n + ray];
    S.lz0[tid] = pb.d[PD_LZ0 * n + ray];
    S.q0[tid] = pb.d[PD_Q0 * n + ray];
    S.local[tid] = local;
#pragma unroll
    for (int j = 0; j < PU_COUNT; ++j) uch[j] = pb.u[j * n + ray];
    double hf, sv;
    const double r = ks_rhs<double>(y, Bp->m, Bp->a, k1, hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        xch[i] = y[i];
        xch[6 + i] = k1[i];
    }
    return r;
}

// Park a ray for the other pass: y and h from xch[0..6], the words in uch[].
template <class ColdT>
__device__ __noinline__ void park_ray(const ParkBuf pb, uint64_t ray, const ColdT& S, int tid,
                                      const double* __restrict__ xch, const uint32_t* __restrict__ uch) {
    const uint64_t n = pb.n;
#pragma unroll
    for (int i = 0; i < 6; ++i) pb.d[(PD_Y + i) * n + ray] = xch[i];
    pb.d[PD_H * n + ray] = xch[6];
    pb.d[PD_LAMBDA * n + ray] = S.lambda[tid];
    pb.d[PD_DH * n + ray] = S.dH[tid];
    pb.d[PD_LZ0 * n + ray] = S.lz0[tid];
    pb.d[PD_Q0 * n + ray] = S.q0[tid];
#pragma unroll
    for (int j = 0; j < PU_COUNT; ++j) pb.u[j * n + ray] = uch[j];
}

// Disk crossing on the continuous extension of an accepted step (near pass of
// the two-pass mixed tracer): Illinois regula falsi on z(t) of the 4th-order
// dense output, which needs no RHS evaluation (the DP5-fraction root of the
// FP64 tracer costs five per iteration).  y0, k1: step start; y1, k7: step
// end; e = h sum_j D_j k_j.  Writes the point at the root to out[0..5] and
// returns t.
__device__ __noinline__ double dense_disk_root(const double* __restrict__ y0, const double* __restrict__ k1,
                                               const double* __restrict__ y1, const double* __restrict__ k7,
                                               const double* __restrict__ e, double h, double* __restrict__ out) {
    double d[6], b[6], c[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        d[i] = y1[i] - y0[i];
        b[i] = h * k1[i] - d[i];
        c[i] = d[i] - h * k7[i] - b[i];
    }
    auto z_at = [&](double t) { return y0[2] + t * (d[2] + (1.0 - t) * (b[2] + t * (c[2] + (1.0 - t) * e[2]))); };
    double lo = 0.0, hi = 1.0, flo = y0[2], fhi = y1[2], t = 1.0;
    int side = 0;
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        const double ft = z_at(t);
        if (ft == 0.0 || fabs(hi - lo) < 1e-15 || fabs(ft) < 1e-13 * (1.0 + fabs(y0[0]) + fabs(y0[1]))) break;
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
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = y0[i] + t * (d[i] + (1.0 - t) * (b[i] + t * (c[i] + (1.0 - t) * e[i])));
    return t;
}

// Record crossing k of a Kerr-Schild ray at the root point yr (winding
// wind_root along the ray) for the translucent-disk continuation: r_BL, the
// unwrapped azimuth and g, as the first hit's record has them.
template <class ColdT>
__device__ __forceinline__ void record_crossing(const TraceArgs& args, const BundleDesc* __restrict__ Bp, ColdT& S,
                                                int j, uint32_t k, const double* __restrict__ yr, int wind_root) {
    const double a = Bp->a;
    const double r = sqrt(bl_r2<double>(yr[0], yr[1], yr[2], a * a));
    const double phi = atan2(yr[1], yr[0]) - atan2(a, r) + kTwoPi * static_cast<double>(wind_root);
    cont_record(args.cont, Bp->out_offset + S.local[j], k, r, phi, disk_redshift(Bp->m, a, r, S.lz0[j]));
}

// End of a Kerr-Schild ray's trace with the continuation on.  xch as end_ray
// takes it: with interp_target > 0 the last step (y0, f0, y1, f1 in xch[0..23],
// length hh), whose end the sky direction is interpolated to the threshold
// radius on; else the ray's last point in xch[0..5].  With the sky on, the end
// goes to the tail record for the shading pass (ks_tail_direction).
template <class ColdT>
__device__ __forceinline__ void end_continuation(const TraceArgs& args, const BundleDesc* __restrict__ Bp, ColdT& S,
                                                 int j, uint32_t n_cross, uint32_t status, const double* __restrict__ xch,
                                                 double interp_target = 0.0, double hh = 0.0) {
    const uint64_t o = Bp->out_offset + S.local[j];
    const double* yl = xch + (interp_target > 0.0 ? 12 : 0);
    if (args.cont.tail) {
        double2* T = reinterpret_cast<double2*>(args.cont.tail + o * TL_COUNT);
        if (interp_target > 0.0) {
#pragma unroll
            for (int i = 0; i < 12; ++i) T[i] = make_double2(xch[2 * i], xch[2 * i + 1]);
        } else {
#pragma unroll
            for (int i = 0; i < 3; ++i) T[TL_Y1 / 2 + i] = make_double2(xch[2 * i], xch[2 * i + 1]);
        }
        T[TL_H / 2] = make_double2(hh, interp_target);
        T[TL_M / 2] = make_double2(Bp->m, Bp->a);
    }
    cont_finish(args.cont, o, n_cross, status, sqrt(bl_r2<double>(yl[0], yl[1], yl[2], Bp->a * Bp->a)), Bp->m);
}

// A ray's end (capture, escape, unfinished): its record and pixel unless it
// crossed the disk before (they describe the first hit, written then), and its
// continuation outputs when the continuation is on.  xch as finish_ray takes
// it; the ray's last point is xch[12..17] with interp_target > 0, else xch[0..5].
template <bool CONT, class ColdT>
__device__ __forceinline__ void end_ray(const TraceArgs& args, const BundleDesc* __restrict__ Bp, ColdT& S, int j,
                                        uint32_t n_cross, uint32_t status, uint32_t flags, uint32_t acc, uint32_t rej,
                                        int wind, double interp_target, double hh, const double* __restrict__ xch) {
    if constexpr (CONT) {
        if (n_cross == 0)
            finish_ray(Bp, S, j, status, flags, acc, rej, wind, interp_target, hh, NAN, 1.0, args.out, xch);
        end_continuation(args, Bp, S, j, n_cross, status, xch, interp_target, hh);
    } else {
        finish_ray(Bp, S, j, status, flags, acc, rej, wind, interp_target, hh, NAN, 1.0, args.out, xch);
    }
}

// A ray in the near pass returns to the far pass once r_BL exceeds this
// multiple of the FP64 radius (hysteresis against ping-pong at the boundary).
constexpr double kNearExitFactor = 1.25;

// Near-critical rays of the mixed tracer: a ray whose impact parameter lies
// within the camera's band (BundleDesc::critical_band, M) of the critical
// curve (|d_b| from the Kerr radial potential, shadow_distance) orbits the
// photon region, where a step error grows about as 1/|d_b|.  The two-pass
// tracer hands such a ray, before its first step, to the critical pass: the
// FP64 kernel over a queue of those rays, at the camera's tolerance times
// critical_tol_scale.  The single-kernel form keeps such a lane in FP64.
constexpr double kCriticalTolScale = 1e-2;  // the smallest tolerance factor

// Tolerance factor of a near-critical ray: (|d_b| / band)^2, at least
// kCriticalTolScale; 1 at the band's edge, where the FP32 stages' error
// already meets the stated bound.
__device__ __forceinline__ float critical_tol_scale(double db, double band) {
    const double u = fabs(db) / band;
    return static_cast<float>(fmin(1.0, fmax(kCriticalTolScale, u * u)));
}

// Largest r_BL at which the FP32 stages are used (keeps r^4 and 1/r^4 in range).
constexpr double kFp32MaxRadius = 1e6;

}  // namespace

}  // namespace relsim
