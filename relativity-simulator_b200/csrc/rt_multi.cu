// rt_multi.cu -- multi-source Kerr-Schild tracer for sm_100a (FP64).
//
// SoftwareComputeEngine's multi-source path (software_compute_engine.hpp:
// 2708-3252): the camera's hole at the origin plus black-hole bodies, each with
// its own mass, spin axis and thin disk.  The ray equations sum every source's
// Kerr-Schild terms evaluated in that source's local frame (ms_rhs :2857-2871);
// they are the Hamiltonian flow of H = (|p|^2 - 1)/2 - sum_i H_i s_i^2
// (s_i = 1 + k_i . p), onto whose zero set each accepted step is projected.
// The reference steps this path with heuristic RK4; here it runs under the
// DP45 + PI30 machinery of the single-hole tracer, with
//   - a step cap from the nearest source, |h| <= c min_i max(r_i - r_+i, 0.01 m_i);
//   - capture inside capture_scale * r_+ of any source, or when |p| exceeds
//     1000 (a horizon-like region of the summed fields, flag DIVERGED);
//   - escape at |x| > escape radius, the terminal point interpolated to it;
//   - a disk hit at the earliest local-equator crossing of a step that lies on
//     that source's disk, solved on the step's 4th-order dense output, with
//     g = redshift_at(m_i, a_i, r, L_z), L_z from the unit local momentum as in
//     trace_multi_source (:3155).
// Sources live in global memory per bundle (at most 16, read through L1 by
// whole warps of one bundle).  The stage loop is rolled around one copy of the
// N-source RHS, its stage derivatives in shared memory.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "rt_device.cuh"
#include "rt_internal.h"

namespace relsim {

namespace {

constexpr double kMsMaxMomentum = 1e3;
constexpr double kTwoPi = 6.283185307179586476925286766559;
enum MsMode : int { MS_IDLE = 0, MS_STEP = 1 };

// Dormand-Prince rows for the rolled step (rk45_adaptive.hpp:196-203): row s
// gives the weights of k1..k(s+1) in the input of stage s + 2; row 5 is the
// 5th-order solution.  kMsE: error weights of k1..k7.
__constant__ double kMsA[6][6] = {
    {DP::A21, 0, 0, 0, 0, 0},
    {DP::A31, DP::A32, 0, 0, 0, 0},
    {DP::A41, DP::A42, DP::A43, 0, 0, 0},
    {DP::A51, DP::A52, DP::A53, DP::A54, 0, 0},
    {DP::A61, DP::A62, DP::A63, DP::A64, DP::A65, 0},
    {DP::B1, 0.0, DP::B3, DP::B4, DP::B5, DP::B6}};
__constant__ double kMsE[7] = {DP::E1, 0.0, DP::E3, DP::E4, DP::E5, DP::E6, DP::E7};
__constant__ double kMsD[7] = {DP::D1, 0.0, DP::D3, DP::D4, DP::D5, DP::D6, DP::D7};

template <int BLOCK>
struct MsCold {
    double k[6][6][BLOCK];  // stage derivatives k2..k7
    double lambda[BLOCK];
    double dH[BLOCK];
    double phi[BLOCK];
    uint64_t local[BLOCK];
};

__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Superposed RHS; returns min_i max(r_i - r_+i, 0.01 m_i) and the first source
// whose local r_BL < capture_scale r_+ (-1: none).
__device__ double ms_rhs(const MsSource* __restrict__ src, uint32_t n, const double* __restrict__ y,
                         double* __restrict__ dy, double cap_scale, int& inside) {
    double cap = 1e300;
    int in = -1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dy[k] = y[3 + k];
        dy[3 + k] = 0.0;
    }
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        const MsSource& s = src[i];
        const double rel[3] = {y[0] - s.pos[0], y[1] - s.pos[1], y[2] - s.pos[2]};
        double ly[6];
        ly[0] = dot3(rel, s.fx);
        ly[1] = dot3(rel, s.fy);
        ly[2] = dot3(rel, s.axis);
        ly[3] = dot3(y + 3, s.fx);
        ly[4] = dot3(y + 3, s.fy);
        ly[5] = dot3(y + 3, s.axis);
        double ld[6], hf, sv;
        const double r = ks_rhs<double, true>(ly, s.m, s.a, ld, hf, sv);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            dy[k] += ld[0] * s.fx[k] + ld[1] * s.fy[k] + ld[2] * s.axis[k];
            dy[3 + k] += ld[3] * s.fx[k] + ld[4] * s.fy[k] + ld[5] * s.axis[k];
        }
        cap = fmin(cap, fmax(r - s.rh, 0.01 * s.m));
        if (in < 0 && r < cap_scale * s.rh) in = static_cast<int>(i);
    }
    inside = in;
    return cap;
}

// Stages 2..7 around one RHS copy; K holds k2..k7 on return.
template <int BLOCK>
__device__ __forceinline__ void ms_stages(const MsSource* __restrict__ src, uint32_t n, const double* __restrict__ y,
                                          const double* __restrict__ k1, double hh, MsCold<BLOCK>& S, int tid,
                                          double cap_scale, double* __restrict__ y5, double* __restrict__ k7,
                                          double* __restrict__ est, double& cap5, int& inside5) {
#pragma unroll 1
    for (int st = 0; st < 6; ++st) {
        double in[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double acc = kMsA[st][0] * k1[i];
#pragma unroll 1
            for (int j = 1; j <= st; ++j) acc += kMsA[st][j] * S.k[j - 1][i][tid];
            in[i] = y[i] + hh * acc;
        }
        if (st == 5) {
#pragma unroll
            for (int i = 0; i < 6; ++i) y5[i] = in[i];
        }
        double out[6];
        int ins;
        const double c = ms_rhs(src, n, in, out, cap_scale, ins);
#pragma unroll
        for (int i = 0; i < 6; ++i) S.k[st][i][tid] = out[i];
        if (st == 5) {
#pragma unroll
            for (int i = 0; i < 6; ++i) k7[i] = out[i];
            cap5 = c;
            inside5 = ins;
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double acc = kMsE[0] * k1[i];
#pragma unroll 1
        for (int j = 2; j < 7; ++j) acc += kMsE[j] * S.k[j - 1][i][tid];
        est[i] = fabs(hh) * fabs(acc);
    }
}

// Coefficients of the step's dense output y(t) = y0 + t (d + (1-t)(b + t(c + (1-t) e))).
template <int BLOCK>
__device__ __forceinline__ void ms_dense_coeffs(const double* __restrict__ y0, const double* __restrict__ y1,
                                                const double* __restrict__ k1, const double* __restrict__ k7, double h,
                                                const MsCold<BLOCK>& S, int tid, double (*co)[6]) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const double d = y1[i] - y0[i];
        const double b = h * k1[i] - d;
        double e = kMsD[0] * k1[i] + kMsD[6] * k7[i];
#pragma unroll 1
        for (int j = 2; j < 6; ++j) e += kMsD[j] * S.k[j - 1][i][tid];
        co[0][i] = d;
        co[1][i] = b;
        co[2][i] = d - h * k7[i] - b;
        co[3][i] = h * e;
    }
}

__device__ __forceinline__ double ms_dense_at(const double* y0, const double (*co)[6], int i, double t) {
    return y0[i] + t * (co[0][i] + (1.0 - t) * (co[1][i] + t * (co[2][i] + (1.0 - t) * co[3][i])));
}

// Illinois root on [0, 1] of the local z of source s on the dense output.
__device__ double ms_local_z_root(const MsSource& s, const double* y0, const double (*co)[6], double f0, double f1) {
    double lo = 0.0, hi = 1.0, flo = f0, fhi = f1, t = 1.0;
    int side = 0;
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        const double rel[3] = {ms_dense_at(y0, co, 0, t) - s.pos[0], ms_dense_at(y0, co, 1, t) - s.pos[1],
                               ms_dense_at(y0, co, 2, t) - s.pos[2]};
        const double ft = dot3(rel, s.axis);
        if (ft == 0.0 || fabs(hi - lo) < 1e-15 || fabs(ft) < 1e-13 * (1.0 + fabs(rel[0]) + fabs(rel[1]))) break;
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

// Fraction of the step where |x| of the cubic Hermite interpolant crosses target.
__device__ double ms_radius_crossing(const double* y0, const double* f0, const double* y1, const double* f1, double h,
                                     double target) {
    double lo = 0.0, hi = 1.0, x[6];
    double flo = sqrt(dot3(y0, y0)) - target, fhi = sqrt(dot3(y1, y1)) - target;
    if (!((flo > 0.0) != (fhi > 0.0))) return 1.0;
    int side = 0;
    double t = 1.0;
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        hermite(y0, f0, y1, f1, h, t, 3, x);
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

// Projection of p onto H = 0 along n = dH/dp, closest root; returns |H| before.
// Two passes over the sources (n needs all of them first).
__device__ double ms_project(const MsSource* __restrict__ src, uint32_t n, double* y, double tol) {
    double* p = y + 3;
    double nv[3] = {p[0], p[1], p[2]};
    double sum = 0.0;
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        const MsSource& s = src[i];
        const double rel[3] = {y[0] - s.pos[0], y[1] - s.pos[1], y[2] - s.pos[2]};
        const double lx[3] = {dot3(rel, s.fx), dot3(rel, s.fy), dot3(rel, s.axis)};
        double kl[3], hf;
        ks_field64(lx, s.m, s.a, kl, hf);
        double kw[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) kw[k] = kl[0] * s.fx[k] + kl[1] * s.fy[k] + kl[2] * s.axis[k];
        const double sv = 1.0 + dot3(kw, p);
        sum += hf * sv * sv;
#pragma unroll
        for (int k = 0; k < 3; ++k) nv[k] -= 2.0 * hf * sv * kw[k];
    }
    const double res = 0.5 * (dot3(p, p) - 1.0) - sum;
    if (!(fabs(res) >= tol)) return fabs(res);
    double qa = 0.5 * dot3(nv, nv), qb = dot3(p, nv);
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        const MsSource& s = src[i];
        const double rel[3] = {y[0] - s.pos[0], y[1] - s.pos[1], y[2] - s.pos[2]};
        const double lx[3] = {dot3(rel, s.fx), dot3(rel, s.fy), dot3(rel, s.axis)};
        double kl[3], hf;
        ks_field64(lx, s.m, s.a, kl, hf);
        double kw[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) kw[k] = kl[0] * s.fx[k] + kl[1] * s.fy[k] + kl[2] * s.axis[k];
        const double sv = 1.0 + dot3(kw, p);
        const double kn = dot3(kw, nv);
        qa -= hf * kn * kn;
        qb -= 2.0 * hf * sv * kn;
    }
    const double disc = qb * qb - 4.0 * qa * res;
    if (disc >= 0.0) {
        const double q = -0.5 * (qb + copysign(sqrt(disc), qb));
        if (q != 0.0) {
            const double alpha = res / q;
#pragma unroll
            for (int k = 0; k < 3; ++k) p[k] += alpha * nv[k];
        }
    }
    return fabs(res);
}

// Static observer's null momentum in the superposed metric (ms_initial_momentum,
// software_compute_engine.hpp:2915-2964).
__device__ __noinline__ void ms_initial_momentum(const MsSource* __restrict__ src, uint32_t n, const double* x,
                                                 const double* outward, double* pout) {
    // potentials and world directions are recomputed where needed (no per-source arrays)
    auto field = [&](uint32_t i, double& pot, double* dir) {
        const MsSource& s = src[i];
        const double rel[3] = {x[0] - s.pos[0], x[1] - s.pos[1], x[2] - s.pos[2]};
        const double lx[3] = {dot3(rel, s.fx), dot3(rel, s.fy), dot3(rel, s.axis)};
        double kl[3];
        ks_field64(lx, s.m, s.a, kl, pot);
#pragma unroll
        for (int k = 0; k < 3; ++k) dir[k] = kl[0] * s.fx[k] + kl[1] * s.fy[k] + kl[2] * s.axis[k];
    };
    auto mdot = [&](const double* a, const double* b) {
        double v = -a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
        for (uint32_t i = 0; i < n; ++i) {
            double pot, dir[3];
            field(i, pot, dir);
            const double la = a[0] + dir[0] * a[1] + dir[1] * a[2] + dir[2] * a[3];
            const double lb = b[0] + dir[0] * b[1] + dir[1] * b[2] + dir[2] * b[3];
            v += 2.0 * pot * la * lb;
        }
        return v;
    };
    double sum = 0.0;
    double e[3][4];
    for (int j = 0; j < 3; ++j) e[j][0] = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        double pot, dir[3];
        field(i, pot, dir);
        sum += pot;
        for (int j = 0; j < 3; ++j) e[j][0] += pot * dir[j];  // shift of axis j
    }
    const double ilsq = 1.0 / fmax(1.0 - 2.0 * sum, 1e-6);
    const double u0 = sqrt(ilsq);
    for (int j = 0; j < 3; ++j) {
        e[j][0] = 2.0 * e[j][0] * ilsq;
        e[j][1] = (j == 0) ? 1.0 : 0.0;
        e[j][2] = (j == 1) ? 1.0 : 0.0;
        e[j][3] = (j == 2) ? 1.0 : 0.0;
    }
    for (int j = 0; j < 3; ++j) {
        double d[2] = {0.0, 0.0};
        for (int q = 0; q < j; ++q) d[q] = mdot(e[j], e[q]);
        for (int q = 0; q < j; ++q)
            for (int c = 0; c < 4; ++c) e[j][c] -= d[q] * e[q][c];
        const double norm = sqrt(fmax(mdot(e[j], e[j]), 1e-30));
        for (int c = 0; c < 4; ++c) e[j][c] /= norm;
    }
    double v[4];
    for (int c = 0; c < 4; ++c) v[c] = -outward[0] * e[0][c] - outward[1] * e[1][c] - outward[2] * e[2][c];
    v[0] += u0;
    double mom[3] = {v[1], v[2], v[3]};
    double tc = -v[0];
    for (uint32_t i = 0; i < n; ++i) {
        double pot, dir[3];
        field(i, pot, dir);
        const double lv = v[0] + dir[0] * v[1] + dir[1] * v[2] + dir[2] * v[3];
        tc += 2.0 * pot * lv;
        for (int k = 0; k < 3; ++k) mom[k] += 2.0 * pot * lv * dir[k];
    }
    const double inv = 1.0 / fmax(-tc, 1e-12);
    for (int k = 0; k < 3; ++k) pout[k] = mom[k] * inv;
}

// Ray generation: pixel -> pinhole direction -> world direction (as the
// single-hole tracer), the observer's Cartesian point, initial momentum.
__device__ __noinline__ void ms_init_ray(const MsDesc* __restrict__ Bp, const MsSource* __restrict__ src,
                                         uint64_t local, double* __restrict__ y) {
    const MsDesc& B = *Bp;
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
    y[0] = B.x0[0];
    y[1] = B.x0[1];
    y[2] = B.x0[2];
    ms_initial_momentum(src, B.src_count, y, d, y + 3);
}

template <int BLOCK>
__device__ __noinline__ void ms_finish(const MsDesc* __restrict__ Bp, const MsSource* __restrict__ src,
                                       MsCold<BLOCK>& S, int tid, const double* y,
                                       uint32_t status, uint32_t flags, uint32_t acc, uint32_t rej, double r_hit,
                                       double g, uint32_t body, const OutPtrs& out) {
    const double r = sqrt(dot3(y, y));
    const double theta = acos(fmin(fmax(y[2] / fmax(r, 1e-300), -1.0), 1.0));
    const uint64_t o = Bp->out_offset + S.local[tid];
    const rt_ray_out& R = out.rays;
    if (R.status) R.status[o] = status;
    if (R.flags) R.flags[o] = flags;
    if (R.steps_accepted) R.steps_accepted[o] = acc;
    if (R.steps_rejected) R.steps_rejected[o] = rej;
    if (R.r) R.r[o] = r;
    if (R.theta) R.theta[o] = theta;
    if (R.phi) R.phi[o] = S.phi[tid];
    if (R.r_hit) R.r_hit[o] = r_hit;
    if (R.g) R.g[o] = g;
    if (R.lambda) R.lambda[o] = S.lambda[tid];
    if (R.dH) R.dH[o] = S.dH[tid];
    if (R.dE) R.dE[o] = NAN;
    if (R.dLz) R.dLz[o] = NAN;
    if (R.dQ) R.dQ[o] = NAN;
    if (R.body) R.body[o] = body;
    if (R.exit_x || R.exit_y || R.exit_z) {
        // sky-lookup direction of an escaped ray: minus the normalised flow of the
        // superposed RHS at the terminal state, (0, 0, -1) where it vanishes
        // (software_compute_engine.hpp:3220-3224)
        double e[3] = {NAN, NAN, NAN};
        if (status == RT_RAY_ESCAPED) {
            double dy[6];
            int ins;
            ms_rhs(src, Bp->src_count, y, dy, Bp->capture_scale, ins);
            const double len = sqrt(dot3(dy, dy));
            if (len > 1e-12) {
#pragma unroll
                for (int i = 0; i < 3; ++i) e[i] = -dy[i] / len;
            } else {
                e[0] = e[1] = 0.0;
                e[2] = -1.0;
            }
        }
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

// Translucent-disk continuation of a multi-source ray (trace_multi_source,
// software_compute_engine.hpp:3150-3191): every disk crossing recorded in
// order along the ray (radius, local azimuth, g and the source), the ray
// followed to its end.  End record: crossings, class at the end, and whether
// the end point lies within 6 m of a source (where the reference drops the
// remaining throughput instead of adding the sky, :3207-3216).
__device__ __forceinline__ void ms_cont_record(const ContOut& C, uint64_t o, uint32_t k, double r, double az,
                                               double g) {
    C.cross[(3 * k) * C.stride + o] = r;
    C.cross[(3 * k + 1) * C.stride + o] = az;
    C.cross[(3 * k + 2) * C.stride + o] = g;
}

__device__ __noinline__ void ms_cont_finish(const ContOut& C, uint64_t o, uint32_t n_cross, uint32_t bodies,
                                            uint32_t status, const MsSource* __restrict__ src, uint32_t n,
                                            const double* x) {
    bool near = false;
    for (uint32_t i = 0; i < n; ++i) {
        const double d[3] = {x[0] - src[i].pos[0], x[1] - src[i].pos[1], x[2] - src[i].pos[2]};
        near = near || sqrt(dot3(d, d)) < 6.0 * src[i].m;
    }
    C.info[o] = n_cross | (status << CI_FATE_SHIFT) | (near ? CI_INSIDE_3RS : 0u);
    C.body[o] = bodies;
    if (C.exit) {
        // the sky-lookup direction at the end: minus the normalised flow of the
        // superposed RHS, (0, 0, -1) where it vanishes (:3220-3224)
        double dy[6], e[3] = {0.0, 0.0, -1.0};
        int ins;
        ms_rhs(src, n, x, dy, 1.0, ins);
        const double len = sqrt(dot3(dy, dy));
        if (len > 1e-12)
            for (int i = 0; i < 3; ++i) e[i] = -dy[i] / len;
        C.exit[o] = e[0];
        C.exit[C.stride + o] = e[1];
        C.exit[2 * C.stride + o] = e[2];
    }
}

__device__ __forceinline__ void ms_unwrap(double& phi, const double* y) {
    double d = atan2(y[1], y[0]) - phi;
    d -= kTwoPi * floor(d / kTwoPi + 0.5);
    phi += d;
}

template <int BLOCK, bool CONT>
__global__ void __launch_bounds__(BLOCK, 384 / BLOCK) ms_trace_kernel(MsArgs args) {
    __shared__ MsCold<BLOCK> S;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const unsigned lt_mask = (1u << lane) - 1u;

    double y[6], k1[6];
    double h = 0.0, cap_len = 0.0;
    float lnp = 0.0f;
    bool has_hist = false;
    int inside = -1;
    uint32_t acc = 0, rej = 0, flags = 0, bidx = 0, guard = 0;
    int mode = MS_IDLE;
    uint32_t n_cross = 0, bodies = 0;  // continuation: crossings so far, their sources
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] = k1[i] = 0.0;
    bool queue_open = true;
    uint64_t chunk_next = 0, chunk_end = 0;
    uint32_t n_att = 0, n_acc = 0, n_rays = 0;

    for (;;) {
        // refill idle lanes from the warp's chunk, then from a new chunk (one atomic)
        const unsigned idle = __ballot_sync(FULL, mode == MS_IDLE);
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
            if (mode == MS_IDLE) {
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
                    const MsDesc* Bp = args.bundles + lo;
                    const MsSource* src = args.sources + Bp->src_begin;
                    S.local[tid] = rid - Bp->ray_begin;
                    ms_init_ray(Bp, src, S.local[tid], y);
                    int ins;
                    cap_len = ms_rhs(src, Bp->src_count, y, k1, Bp->capture_scale, ins);
                    inside = ins;
                    h = -Bp->h0;
                    lnp = 0.0f;
                    has_hist = false;
                    acc = rej = flags = guard = 0;
                    S.lambda[tid] = 0.0;
                    S.dH[tid] = 0.0;
                    S.phi[tid] = Bp->phi0;
                    n_cross = bodies = 0;
                    mode = MS_STEP;
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
        if (__ballot_sync(FULL, mode != MS_IDLE) == 0) {
            if (!queue_open && chunk_next >= chunk_end) break;
            continue;
        }
        if (mode == MS_IDLE) continue;

        const MsDesc* Bp = args.bundles + bidx;
        const MsSource* src = args.sources + Bp->src_begin;
        const uint32_t ns = Bp->src_count;
        // the end of a ray: its record (with the continuation only when it crossed
        // no disk: the record describes the first hit) and its continuation end
        auto end_ray = [&](const double* yend, uint32_t status, uint32_t fl, uint32_t body) {
            if (!CONT || n_cross == 0)
                ms_finish<BLOCK>(Bp, src, S, tid, yend, status, fl, acc, rej, NAN, 1.0, body, args.out);
            if constexpr (CONT)
                ms_cont_finish(args.cont, Bp->out_offset + S.local[tid], n_cross, bodies, status, src, ns, yend);
            mode = MS_IDLE;
        };
        // backstop on loop iterations per ray (one attempt per iteration)
        uint32_t term = 0;
        if (++guard > Bp->max_steps + 64u) {
            flags |= RT_RAYFLAG_MAX_STEPS;
            term = RT_RAY_UNFINISHED + 16;
        } else if (inside >= 0) {
            term = RT_RAY_CAPTURED;
        } else if (dot3(y + 3, y + 3) > kMsMaxMomentum * kMsMaxMomentum) {
            flags |= RT_RAYFLAG_DIVERGED;
            term = RT_RAY_CAPTURED;
        } else if (dot3(y, y) > Bp->r_esc * Bp->r_esc) {
            term = RT_RAY_ESCAPED;
        } else if (acc + rej >= Bp->max_steps) {
            flags |= RT_RAYFLAG_MAX_STEPS;
            term = RT_RAY_UNFINISHED + 16;
        } else {
            const double cap = Bp->cap_c * cap_len;
            if (fabs(h) > cap) h = -cap;
            if (fabs(h) < 1e-8) {
                flags |= RT_RAYFLAG_STEP_UNDERFLOW;
                term = RT_RAY_CAPTURED;
            }
        }
        if (term) {
            const uint32_t cls = term & 15u;
            end_ray(y, cls, flags,
                    (cls == RT_RAY_CAPTURED && inside >= 0) ? static_cast<uint32_t>(inside) : RT_BODY_NONE);
            continue;
        }

        const double hh = h;
        double y5[6], k7[6], est[6], cap5;
        int inside5;
        ms_stages<BLOCK>(src, ns, y, k1, hh, S, tid, Bp->capture_scale, y5, k7, est, cap5, inside5);
        double err;
        {
            double num = 0.0, den = 1.0;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const double sc = Bp->rtol * fmax(fabs(y[i]), fabs(y5[i])) + Bp->atol;
                if (est[i] * den > num * sc) {
                    num = est[i];
                    den = sc;
                }
            }
            err = num / den;
        }
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
        bool finite = true;
#pragma unroll
        for (int i = 0; i < 6; ++i) finite = finite && isfinite(y5[i]);
        if (!finite) {
            end_ray(y, RT_RAY_CAPTURED, flags | RT_RAYFLAG_NONFINITE, RT_BODY_NONE);
            continue;
        }
        // disk crossings of this step in order along the ray, each the earliest
        // local-equator crossing on a disk after the previous one: the first ends
        // the ray; under the continuation each is recorded and the ray goes on
        {
            bool ended = false;
            double t_prev = -1.0;
#pragma unroll 1
            for (uint32_t pass = 0; pass < ns; ++pass) {
                double best = 2.0, best_r = 0.0, best_lz = 0.0, best_az = 0.0;
                uint32_t best_i = 0;
#pragma unroll 1
                for (uint32_t i = 0; i < ns; ++i) {
                    const MsSource& s = src[i];
                    if (s.disk_in < 0.0) continue;
                    const double r0[3] = {y[0] - s.pos[0], y[1] - s.pos[1], y[2] - s.pos[2]};
                    const double r1[3] = {y5[0] - s.pos[0], y5[1] - s.pos[1], y5[2] - s.pos[2]};
                    const double z0 = dot3(r0, s.axis), z1 = dot3(r1, s.axis);
                    if (!(z0 * z1 <= 0.0) || z0 == z1) continue;
                    const double sl = z0 / (z0 - z1);
                    const double ce[3] = {r0[0] + sl * (r1[0] - r0[0]), r0[1] + sl * (r1[1] - r0[1]),
                                          r0[2] + sl * (r1[2] - r0[2])};
                    const double lxe = dot3(ce, s.fx), lye = dot3(ce, s.fy);
                    const double re = sqrt(fmax(lxe * lxe + lye * lye - s.a * s.a, 0.0));
                    const double margin = 0.05 * re + 0.5 * s.m;
                    if (re < s.disk_in - margin || re > s.disk_out + margin) continue;
                    double co[4][6];
                    ms_dense_coeffs<BLOCK>(y, y5, k1, k7, hh, S, tid, co);
                    const double t = ms_local_z_root(s, y, co, z0, z1);
                    if (!(t < best) || !(t > t_prev)) continue;
                    double yr[6];
#pragma unroll
                    for (int q = 0; q < 6; ++q) yr[q] = ms_dense_at(y, co, q, t);
                    const double rel[3] = {yr[0] - s.pos[0], yr[1] - s.pos[1], yr[2] - s.pos[2]};
                    const double c0 = dot3(rel, s.fx), c1 = dot3(rel, s.fy);
                    const double pl[3] = {dot3(yr + 3, s.fx), dot3(yr + 3, s.fy), dot3(yr + 3, s.axis)};
                    const double rr = sqrt(fmax(c0 * c0 + c1 * c1 - s.a * s.a, 0.0));
                    if (rr < s.disk_in || rr > s.disk_out || rr <= s.rh * 1.02) continue;
                    best = t;
                    best_r = rr;
                    best_i = i;
                    best_lz = (c0 * pl[1] - c1 * pl[0]) / fmax(sqrt(dot3(pl, pl)), 1e-30);
                    // local azimuth of the crossing (ms_disk_crossing, :3037)
                    best_az = atan2(c1, c0) - atan2(s.a, rr);
                }
                if (best > 1.0) break;
                double co[4][6], yr[6];
                ms_dense_coeffs<BLOCK>(y, y5, k1, k7, hh, S, tid, co);
#pragma unroll
                for (int q = 0; q < 6; ++q) yr[q] = ms_dense_at(y, co, q, best);
                const MsSource& s = src[best_i];
                const double g = disk_redshift(s.m, s.a, best_r, best_lz);
                const double lam = S.lambda[tid], ph0 = S.phi[tid];
                if (!CONT || n_cross == 0) {
                    S.lambda[tid] = lam + best * hh;
                    double ph = ph0;
                    ms_unwrap(ph, yr);
                    S.phi[tid] = ph;
                    ms_finish<BLOCK>(Bp, src, S, tid, yr, RT_RAY_DISK, flags, acc, rej, best_r, g, best_i, args.out);
                }
                if constexpr (!CONT) {
                    mode = MS_IDLE;
                    ended = true;
                    break;
                } else {
                    // the crossing recorded; the ray goes on through the disk
                    S.lambda[tid] = lam;
                    S.phi[tid] = ph0;
                    ms_cont_record(args.cont, Bp->out_offset + S.local[tid], n_cross, best_r, best_az, g);
                    bodies |= best_i << (4u * n_cross);
                    ++n_cross;
                    t_prev = best;
                    if (n_cross >= kMaxCrossings) {
                        ms_cont_finish(args.cont, Bp->out_offset + S.local[tid], n_cross, bodies, RT_RAY_UNFINISHED,
                                       src, ns, yr);
                        mode = MS_IDLE;
                        ended = true;
                        break;
                    }
                }
            }
            if (ended) continue;
        }
        if (inside5 >= 0) {  // captured inside this step: its end point
            S.lambda[tid] += hh;
            double ph = S.phi[tid];
            ms_unwrap(ph, y5);
            S.phi[tid] = ph;
            end_ray(y5, RT_RAY_CAPTURED, flags, static_cast<uint32_t>(inside5));
            continue;
        }
        if (dot3(y5, y5) > Bp->r_esc * Bp->r_esc) {  // escaped: interpolated to the escape radius
            const double t = ms_radius_crossing(y, k1, y5, k7, hh, Bp->r_esc);
            double yt[6];
            hermite(y, k1, y5, k7, hh, t, 6, yt);
            S.lambda[tid] += t * hh;
            double ph = S.phi[tid];
            ms_unwrap(ph, yt);
            S.phi[tid] = ph;
            end_ray(yt, RT_RAY_ESCAPED, flags, RT_BODY_NONE);
            continue;
        }
        S.dH[tid] = fmax(S.dH[tid], ms_project(src, ns, y5, Bp->proj_tol));
        {
            double ph = S.phi[tid];
            ms_unwrap(ph, y5);
            S.phi[tid] = ph;
        }
        S.lambda[tid] += hh;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            y[i] = y5[i];
            k1[i] = k7[i];
        }
        cap_len = cap5;
        inside = inside5;
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

template __global__ void ms_trace_kernel<128, false>(MsArgs);
template __global__ void ms_trace_kernel<128, true>(MsArgs);

}  // namespace

uint32_t ms_trace_grid(int sm_count) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ms_trace_kernel<128, false>, 128, 0) != cudaSuccess) {
        cudaGetLastError();
        occ = 1;
    }
    return static_cast<uint32_t>(sm_count) * static_cast<uint32_t>(occ > 1 ? occ : 1);
}

void launch_ms_trace(const MsArgs& args, uint32_t grid, void* stream) {
    if (args.cont.cross)
        ms_trace_kernel<128, true><<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(args);
    else
        ms_trace_kernel<128, false><<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(args);
}

}  // namespace relsim
