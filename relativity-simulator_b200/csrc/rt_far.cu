// rt_far.cu -- far pass of the two-pass mixed-precision tracer, two rays per
// thread.
//
// The far zone (r_BL >= the FP64 radius) is where the mixed tracer spends
// about nine tenths of its step attempts.  There the six new Dormand-Prince
// stages of an attempt run in FP32 on the deviation from free streaming (see
// far_stages); the state, the 5th-order solution, the step-size error norm,
// the H = 0 projection and every decision stay FP64, per ray.  This kernel
// holds two rays per thread ("slots") and evaluates their FP32 stages together
// in Blackwell's packed FP32 arithmetic (fma/mul/add.rn.f32x2): each packed
// instruction computes one operation of both rays, component by component,
// with the rounding of the scalar operation, so a ray's arithmetic is the
// same in either slot and whatever ray shares its thread.  A packed
// instruction does two rays' work in one issue slot, which leaves issue slots
// for the FP64, conversion and control instructions of the step.
//
// The protocol is the single-slot far pass's (rt_trace.cu, PASS_FAR): rays
// start at their pixels (first round) or resume from the far queue; a ray
// that enters the FP64 zone is parked for the near pass; a disk hit is parked
// with its root point for the finish pass; captured, escaped and unfinished
// rays are written here.  A step that crosses z = 0 near the disk is taken
// again in FP64 (stages, dense output, Illinois root on the continuous
// extension), out of line.
//
// The FSAL stage is kept in FP32 form between attempts (its position part as
// the deviation from p), so an attempt converts only the state (6 values),
// the two increments of the 5th-order solution (6) and the error estimate (6)
// between FP64 and FP32.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "rt_device.cuh"
#include "rt_internal.h"
#include "rt_ray.cuh"

namespace relsim {

namespace {

constexpr int kSlots = 2;  // rays per thread

// ---- packed FP32 (f32x2) arithmetic: component s of a float2 belongs to slot s ----
__device__ __forceinline__ float2 bc(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b, rounded once (b * -1 is exact)
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 rsqrt2(float2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
__device__ __forceinline__ float2 max2(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ float lane_of(float2 v, int s) { return s == 0 ? v.x : v.y; }
__device__ __forceinline__ void set_lane(float2& v, int s, float x) {
    if (s == 0) v.x = x;
    else v.y = x;
}

// Kerr-Schild RHS of two rays (the factored form of ks_rhs in rt_device.cuh,
// kerr_schild_null_integrator.hpp:72-114): the gravitational part -2 H s k of
// dx/dlambda and all of dp/dlambda.  a2 = a^2.  Returns r_BL; H and s = 1 + k.p
// through hf, sv.
__device__ __forceinline__ float2 ks_rhs_pair(const float2* __restrict__ in, float2 M, float2 a, float2 a2,
                                              float2* __restrict__ dy, float2& hf, float2& sv) {
    const float2 x = in[0], yy = in[1], z = in[2], px = in[3], py = in[4], pz = in[5];
    const float2 z2 = mul2(z, z);
    const float2 a2z2 = mul2(a2, z2);
    // r_BL^2 = (d + sqrt(d^2 + 4 a^2 z^2)) / 2, d = x^2 + y^2 + z^2 - a^2
    const float2 d = sub2(fma2(x, x, fma2(yy, yy, z2)), a2);
    const float2 w = max2(fma2(d, d, mul2(bc(4.0f), a2z2)), bc(1e-30f));
    const float2 r2 = max2(mul2(bc(0.5f), fma2(w, rsqrt2(w), d)), bc(1e-24f));
    const float2 inv_r = rsqrt2(r2);
    const float2 r = mul2(r2, inv_r);
    const float2 rpa = add2(r2, a2);
    const float2 r4 = mul2(r2, r2);
    const float2 den = add2(r4, a2z2);
    const float2 inv_rpa = rcp2(rpa);
    const float2 inv_den = rcp2(den);
    const float2 r3 = mul2(r2, r);
    const float2 r3d = mul2(r3, inv_den);
    const float2 H = mul2(M, r3d);
    const float2 k0 = mul2(fma2(r, x, mul2(a, yy)), inv_rpa);
    const float2 k1 = mul2(sub2(mul2(r, yy), mul2(a, x)), inv_rpa);
    const float2 k2 = mul2(z, inv_r);
    const float2 s = fma2(k0, px, fma2(k1, py, fma2(k2, pz, bc(1.0f))));
    const float2 hs = mul2(H, s);
    const float2 two_hs = add2(hs, hs);
    const float2 m_two_hs = mul2(bc(-2.0f), hs);
    dy[0] = mul2(m_two_hs, k0);
    dy[1] = mul2(m_two_hs, k1);
    dy[2] = mul2(m_two_hs, k2);
    const float2 dr0 = mul2(r3d, x);
    const float2 dr1 = mul2(r3d, yy);
    const float2 dr2 = mul2(mul2(r, rpa), mul2(z, inv_den));
    // C = M r^2 (3 a^2 z^2 - r^4) / den^2, D = -2 M a^2 r^3 z / den^2 (grouped as in ks_rhs)
    const float2 C = mul2(mul2(M, mul2(r2, inv_den)), mul2(sub2(mul2(bc(3.0f), a2z2), r4), inv_den));
    const float2 D = mul2(mul2(bc(-2.0f), H), mul2(mul2(a2, z), inv_den));
    const float2 m2r = mul2(bc(-2.0f), r);
    const float2 A = sub2(mul2(inv_rpa, fma2(fma2(m2r, k0, x), px, mul2(fma2(m2r, k1, yy), py))),
                          mul2(mul2(inv_r, k2), pz));
    const float2 B0 = mul2(inv_rpa, sub2(mul2(r, px), mul2(a, py)));
    const float2 B1 = mul2(inv_rpa, fma2(r, py, mul2(a, px)));
    const float2 B2 = mul2(inv_r, pz);
    const float2 s2 = mul2(s, s);
    const float2 G = fma2(s2, C, mul2(two_hs, A));
    dy[3] = fma2(dr0, G, mul2(two_hs, B0));
    dy[4] = fma2(dr1, G, mul2(two_hs, B1));
    dy[5] = fma2(dr2, G, fma2(two_hs, B2, mul2(s2, D)));
    hf = H;
    sv = s;
    return r;
}

// FP32 stages of one attempt of two rays.  With x0, p0 the FP32 image of the
// state and dx1, kp1 the FSAL stage (position part minus p, momentum part):
//   x_j = x + h c_j p + h sum_m a_jm dx_m,  dx_m = (p_m - p) - 2 H s k at stage m
//   p_j = p + h sum_m a_jm kp_m
// so the large h p term of every position increment stays with the FP64
// state.  Outputs the FP32 increments of the 5th-order solution
// (y5 = y + h p + incx, p5 = p + incp), the error estimate h sum_j e_j k_j
// (sum_j e_j = 0 puts dx_j in place of the position derivatives), and the
// FSAL stage at the FP32 image of y5: its gravitational position part g7,
// momentum part kp7, and r_BL, H, s there.
__device__ __forceinline__ void far_stages(const float2* __restrict__ x0, const float2* __restrict__ p0,
                                           const float2* __restrict__ dx1, const float2* __restrict__ kp1,
                                           float2 h, float2 M, float2 a, float2 a2, float2* __restrict__ incx,
                                           float2* __restrict__ incp, float2* __restrict__ ex,
                                           float2* __restrict__ ep, float2* __restrict__ g7, float2* __restrict__ kp7,
                                           float2& r7, float2& hf7, float2& s7) {
    float2 dx2[3], kp2[3], dx3[3], kp3[3], dx4[3], kp4[3], dx5[3], kp5[3], dx6[3], kp6[3];
    float2 in[6], g[6], dp[3], hf, sv;
#define RT_PSTAGE(DXO, KPO, CC, SUMX, SUMP)                     \
    _Pragma("unroll") for (int i = 0; i < 3; ++i) {            \
        dp[i] = mul2(h, (SUMP));                               \
        in[i] = fma2(h, fma2(bc(CC), p0[i], (SUMX)), x0[i]);   \
        in[3 + i] = add2(p0[i], dp[i]);                        \
    }                                                          \
    ks_rhs_pair(in, M, a, a2, g, hf, sv);                      \
    _Pragma("unroll") for (int i = 0; i < 3; ++i) {            \
        DXO[i] = add2(dp[i], g[i]);                            \
        KPO[i] = g[3 + i];                                     \
    }
#define C_(v) bc(static_cast<float>(DP::v))
    RT_PSTAGE(dx2, kp2, 0.2f, mul2(C_(A21), dx1[i]), mul2(C_(A21), kp1[i]))
    RT_PSTAGE(dx3, kp3, 0.3f, fma2(C_(A31), dx1[i], mul2(C_(A32), dx2[i])),
              fma2(C_(A31), kp1[i], mul2(C_(A32), kp2[i])))
    RT_PSTAGE(dx4, kp4, 0.8f, fma2(C_(A41), dx1[i], fma2(C_(A42), dx2[i], mul2(C_(A43), dx3[i]))),
              fma2(C_(A41), kp1[i], fma2(C_(A42), kp2[i], mul2(C_(A43), kp3[i]))))
    RT_PSTAGE(dx5, kp5, 8.0f / 9.0f,
              fma2(C_(A51), dx1[i], fma2(C_(A52), dx2[i], fma2(C_(A53), dx3[i], mul2(C_(A54), dx4[i])))),
              fma2(C_(A51), kp1[i], fma2(C_(A52), kp2[i], fma2(C_(A53), kp3[i], mul2(C_(A54), kp4[i])))))
    RT_PSTAGE(dx6, kp6, 1.0f,
              fma2(C_(A61), dx1[i],
                   fma2(C_(A62), dx2[i], fma2(C_(A63), dx3[i], fma2(C_(A64), dx4[i], mul2(C_(A65), dx5[i]))))),
              fma2(C_(A61), kp1[i],
                   fma2(C_(A62), kp2[i], fma2(C_(A63), kp3[i], fma2(C_(A64), kp4[i], mul2(C_(A65), kp5[i]))))))
#undef RT_PSTAGE
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float2 sx = fma2(C_(B1), dx1[i],
                               fma2(C_(B3), dx3[i], fma2(C_(B4), dx4[i], fma2(C_(B5), dx5[i], mul2(C_(B6), dx6[i])))));
        const float2 sp = fma2(C_(B1), kp1[i],
                               fma2(C_(B3), kp3[i], fma2(C_(B4), kp4[i], fma2(C_(B5), kp5[i], mul2(C_(B6), kp6[i])))));
        incx[i] = mul2(h, sx);
        incp[i] = mul2(h, sp);
        // stage 7 input: the FP32 image of y5
        in[i] = add2(x0[i], fma2(h, p0[i], incx[i]));
        in[3 + i] = add2(p0[i], incp[i]);
    }
    r7 = ks_rhs_pair(in, M, a, a2, g, hf7, s7);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        g7[i] = g[i];
        kp7[i] = g[3 + i];
        const float2 dx7 = add2(incp[i], g[i]);
        const float2 sx = fma2(C_(E1), dx1[i],
                               fma2(C_(E3), dx3[i],
                                    fma2(C_(E4), dx4[i], fma2(C_(E5), dx5[i], fma2(C_(E6), dx6[i], mul2(C_(E7), dx7))))));
        const float2 sp =
            fma2(C_(E1), kp1[i],
                 fma2(C_(E3), kp3[i], fma2(C_(E4), kp4[i], fma2(C_(E5), kp5[i], fma2(C_(E6), kp6[i], mul2(C_(E7), g[3 + i]))))));
        ex[i] = mul2(h, sx);
        ep[i] = mul2(h, sp);
    }
#undef C_
}

// A far-zone step that crosses z = 0 near the disk, taken again in FP64: the
// FSAL stage recomputed at y, the six stages, the dense-output term and the
// crossing solved on the continuous extension (dense_disk_root), as the near
// pass does.  Returns r_hit > 0 on a hit, with the root point in out[0..5] and
// its step fraction in out[6]; otherwise -1, with the FP64 step's y5 in
// out[0..5], its FSAL stage k7 in out[6..11] and r_BL, H, s at y5 in
// out[12..14].
__device__ __noinline__ double far_disk_step(const BundleDesc* __restrict__ Bp, const double* __restrict__ y,
                                             double hh, double* __restrict__ out) {
    const double M = Bp->m, a = Bp->a;
    double k1[6], k2[6], k3[6], k4[6], k5[6], k6[6], k7[6], in[6], y5[6], dense[6], hf, sv, hf5, s5;
    ks_rhs<double>(y, M, a, k1, hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i) in[i] = y[i] + hh * (DP::A21 * k1[i]);
    ks_rhs<double>(in, M, a, k2, hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i) in[i] = y[i] + hh * (DP::A31 * k1[i] + DP::A32 * k2[i]);
    ks_rhs<double>(in, M, a, k3, hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i) in[i] = y[i] + hh * (DP::A41 * k1[i] + DP::A42 * k2[i] + DP::A43 * k3[i]);
    ks_rhs<double>(in, M, a, k4, hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i)
        in[i] = y[i] + hh * (DP::A51 * k1[i] + DP::A52 * k2[i] + DP::A53 * k3[i] + DP::A54 * k4[i]);
    ks_rhs<double>(in, M, a, k5, hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i)
        in[i] = y[i] + hh * (DP::A61 * k1[i] + DP::A62 * k2[i] + DP::A63 * k3[i] + DP::A64 * k4[i] + DP::A65 * k5[i]);
    ks_rhs<double>(in, M, a, k6, hf, sv);
#pragma unroll
    for (int i = 0; i < 6; ++i)
        y5[i] = y[i] + hh * (DP::B1 * k1[i] + DP::B3 * k3[i] + DP::B4 * k4[i] + DP::B5 * k5[i] + DP::B6 * k6[i]);
    const double r5 = ks_rhs<double>(y5, M, a, k7, hf5, s5);
#pragma unroll
    for (int i = 0; i < 6; ++i)
        dense[i] = hh * (DP::D1 * k1[i] + DP::D3 * k3[i] + DP::D4 * k4[i] + DP::D5 * k5[i] + DP::D6 * k6[i] +
                         DP::D7 * k7[i]);
    double root[6];
    const double t = dense_disk_root(y, k1, y5, k7, dense, hh, root);
    const double rr = sqrt(bl_r2<double>(root[0], root[1], root[2], a * a));
    if (rr >= Bp->r_in && rr <= Bp->r_out && rr > Bp->rh * 1.02) {
#pragma unroll
        for (int i = 0; i < 6; ++i) out[i] = root[i];
        out[6] = t;
        return rr;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        out[i] = y5[i];
        out[6 + i] = k7[i];
    }
    out[12] = r5;
    out[13] = hf5;
    out[14] = s5;
    return -1.0;
}

// Per-slot ray state held in registers (indexed by compile-time slot numbers
// only, after unrolling).
struct SlotState {
    double y[6];
    double h;
    float r;      // r_BL at y (FP32: far-zone decisions only)
    float lnp;    // log2 of the previous error (PI30 history)
    uint32_t acc, rej, flags, guard, bidx, ray;
    int mode, wind, can_early;
    bool has_hist;
    bool critical;  // near-critical: goes to the FP64 near pass at its first step
};

}  // namespace

// The far pass with two rays per thread.  WARPS_PER_SM * 32 / BLOCK resident
// CTAs per SM: 12 warps cap it at 168 registers per thread (768 rays per SM),
// 8 warps at 255.
template <int BLOCK, int WARPS_PER_SM>
__global__ void __launch_bounds__(BLOCK, WARPS_PER_SM * 32 / BLOCK) far_pair_kernel(TraceArgs args) {
    __shared__ ColdSlots<kSlots * BLOCK> S;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const bool from_queue = args.from_pixels == 0u;
    const uint64_t total = from_queue ? static_cast<uint64_t>(*args.in_count) : args.total_rays;
    // claims and refills count ray slots: 64 per warp
    const uint64_t claim = 2ull * args.claim;
    const int threshold = static_cast<int>(2u * args.refill_threshold < 64u ? 2u * args.refill_threshold : 64u);

    SlotState st[kSlots];
    float2 dx1[3], kp1[3];  // FSAL stage per slot
    float2 Mf = bc(1.0f), af = bc(0.0f), a2f = bc(0.0f);
#pragma unroll
    for (int s = 0; s < kSlots; ++s) {
#pragma unroll
        for (int i = 0; i < 6; ++i) st[s].y[i] = 0.0;
        st[s].h = 0.0;
        st[s].r = 0.0f;
        st[s].lnp = 0.0f;
        st[s].acc = st[s].rej = st[s].flags = st[s].guard = st[s].bidx = st[s].ray = 0u;
        st[s].mode = MODE_IDLE;
        st[s].wind = st[s].can_early = 0;
        st[s].has_hist = false;
        st[s].critical = false;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) dx1[i] = kp1[i] = bc(0.0f);

    bool queue_open = true;
    uint64_t chunk_next = 0, chunk_end = 0;
    uint32_t n_att = 0, n_acc = 0, n_rays = 0, n_rhs = 0, n_redo = 0;

    for (;;) {
        // ---- park the rays that go to the near pass, queue the disk hits ----
        {
            unsigned pm[kSlots], fm[kSlots];
#pragma unroll
            for (int s = 0; s < kSlots; ++s) {
                pm[s] = __ballot_sync(FULL, st[s].mode == MODE_PARK);
                fm[s] = __ballot_sync(FULL, st[s].mode == MODE_FINISHQ);
            }
            const uint32_t np = __popc(pm[0]) + __popc(pm[1]);
            const uint32_t nf = __popc(fm[0]) + __popc(fm[1]);
            if (np | nf) {
                uint32_t pbase = 0, fbase = 0;
                if (lane == 0) {
                    if (np) pbase = atomicAdd(args.out_count, np);
                    if (nf) fbase = atomicAdd(args.finish_count, nf);
                }
                pbase = __shfl_sync(FULL, pbase, 0);
                fbase = __shfl_sync(FULL, fbase, 0);
#pragma unroll
                for (int s = 0; s < kSlots; ++s) {
                    const int m = st[s].mode;
                    if (m == MODE_PARK || m == MODE_FINISHQ) {
                        const unsigned* mk = (m == MODE_PARK) ? pm : fm;
                        const uint32_t rank = (s == 0) ? __popc(mk[0] & lt_mask)
                                                       : __popc(mk[0]) + __popc(mk[1] & lt_mask);
                        if (m == MODE_PARK) args.out_queue[pbase + rank] = st[s].ray;
                        else args.finish_queue[fbase + rank] = st[s].ray;
                        double xch[7];
#pragma unroll
                        for (int i = 0; i < 6; ++i) xch[i] = st[s].y[i];
                        xch[6] = st[s].h;
                        const uint32_t misc = (st[s].has_hist ? PM_HAS_HIST : 0u) |
                                              (static_cast<uint32_t>(st[s].can_early + 1) << PM_EARLY_SHIFT) |
                                              (st[s].critical ? PM_CRITICAL : 0u);
                        const uint32_t uch[PU_COUNT] = {st[s].acc,   st[s].rej,  st[s].flags,
                                                        st[s].guard, static_cast<uint32_t>(st[s].wind),
                                                        misc,        __float_as_uint(st[s].lnp)};
                        park_ray(args.park, st[s].ray, S, tid + s * BLOCK, xch, uch);
                        st[s].mode = MODE_IDLE;
                    }
                }
            }
        }
        // ---- refill idle slots: from the warp's chunk, then a new chunk ----
        {
            unsigned idle[kSlots];
#pragma unroll
            for (int s = 0; s < kSlots; ++s) idle[s] = __ballot_sync(FULL, st[s].mode == MODE_IDLE);
            const int n_idle = __popc(idle[0]) + __popc(idle[1]);
            if ((queue_open || chunk_next < chunk_end) && n_idle > 0 && (n_idle >= threshold || n_idle == 64)) {
                const uint64_t avail = chunk_end - chunk_next;
                uint64_t base2 = 0;
                bool got2 = false;
                if (avail < static_cast<uint64_t>(n_idle) && queue_open) {
                    unsigned long long b = 0;
                    if (lane == 0) b = atomicAdd(args.queue, static_cast<unsigned long long>(claim));
                    b = __shfl_sync(FULL, b, 0);
                    if (b >= total) {
                        queue_open = false;
                    } else {
                        base2 = b;
                        got2 = true;
                        if (b + claim >= total) queue_open = false;
                    }
                }
                const uint64_t used_old = (avail < static_cast<uint64_t>(n_idle)) ? avail : n_idle;
#pragma unroll
                for (int s = 0; s < kSlots; ++s) {
                    if (st[s].mode != MODE_IDLE) continue;
                    const uint64_t rank = (s == 0) ? __popc(idle[0] & lt_mask)
                                                   : __popc(idle[0]) + __popc(idle[1] & lt_mask);
                    uint64_t rid = ~0ull;
                    if (rank < avail) rid = chunk_next + rank;
                    else if (got2) rid = base2 + (rank - avail);
                    if (rid >= total) continue;
                    const uint64_t rix = from_queue ? static_cast<uint64_t>(args.in_queue[rid]) : args.ray_base + rid;
                    uint32_t lo = 0, hi = args.n_bundles;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (args.bundles[mid].ray_begin <= rix) lo = mid; else hi = mid;
                    }
                    const BundleDesc* Bp = args.bundles + lo;
                    SlotState& q = st[s];
                    q.bidx = lo;
                    q.ray = static_cast<uint32_t>(rix);
                    double xch[13];
                    if (from_queue) {
                        uint32_t uch[PU_COUNT];
                        q.r = static_cast<float>(
                            resume_ray(Bp, args.park, rix, rix - Bp->ray_begin, S, tid + s * BLOCK, xch, uch));
                        q.h = xch[12];
                        q.acc = uch[PU_ACC];
                        q.rej = uch[PU_REJ];
                        q.flags = uch[PU_FLAGS];
                        q.guard = uch[PU_GUARD];
                        q.wind = static_cast<int>(uch[PU_WIND]);
                        q.has_hist = (uch[PU_MISC] & PM_HAS_HIST) != 0u;
                        q.can_early = static_cast<int>((uch[PU_MISC] >> PM_EARLY_SHIFT) & 3u) - 1;
                        q.lnp = __uint_as_float(uch[PU_LNP]);
                        q.critical = false;
                    } else {
                        const InitResult ir = init_ray(Bp, rix - Bp->ray_begin, S, tid + s * BLOCK, xch);
                        q.r = static_cast<float>(ir.r);
                        q.can_early = ir.can_early;
                        q.h = -Bp->h0;
                        q.lnp = 0.0f;
                        q.has_hist = false;
                        q.acc = q.rej = q.flags = 0u;
                        q.wind = Bp->wind0;
                        q.guard = 0u;
                        q.critical = false;
                        if (args.opts & TO_CRITICAL_FP64) {
                            // distance of the ray's constants from the critical curve; the
                            // Carter early-capture decision comes from the same value
                            const double db = shadow_distance(Bp->m, Bp->a, 0.0, Bp->rh, S.lz0[tid + s * BLOCK],
                                                              S.q0[tid + s * BLOCK]);
                            if (q.can_early < 0) q.can_early = db > kEarlyCaptureMargin;
                            q.critical = fabs(db) < kCriticalBand * Bp->m;
                        }
                        ++n_rays;
                    }
                    ++n_rhs;
#pragma unroll
                    for (int i = 0; i < 6; ++i) q.y[i] = xch[i];
                    // FSAL stage in FP32 form
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        set_lane(dx1[i], s, static_cast<float>(xch[6 + i] - xch[3 + i]));
                        set_lane(kp1[i], s, static_cast<float>(xch[9 + i]));
                    }
                    const float am = static_cast<float>(Bp->a);
                    set_lane(Mf, s, static_cast<float>(Bp->m));
                    set_lane(af, s, am);
                    set_lane(a2f, s, am * am);
                    q.mode = MODE_STEP;
                }
                if (got2) {
                    chunk_next = base2 + (static_cast<uint64_t>(n_idle) - used_old);
                    chunk_end = base2 + claim;
                    if (chunk_end > total) chunk_end = total;
                } else {
                    chunk_next += used_old;
                }
            }
            if (__ballot_sync(FULL, st[0].mode != MODE_IDLE || st[1].mode != MODE_IDLE) == 0) {
                if (!queue_open && chunk_next >= chunk_end) break;
                continue;
            }
        }

        // ---- per slot: attempt budget, domain, step cap, zone ----
        bool act[kSlots];
#pragma unroll
        for (int s = 0; s < kSlots; ++s) {
            SlotState& q = st[s];
            act[s] = false;
            if (q.mode != MODE_STEP) continue;
            const BundleDesc* Bp = args.bundles + q.bidx;
            const double r = static_cast<double>(q.r);
            // order of the single-slot pass: the iteration backstop, the domain, the
            // attempt budget, the step cap, then the zone
            uint32_t term = 0;
            if (++q.guard > 64u * Bp->max_steps + 64u) {
                q.flags |= RT_RAYFLAG_MAX_STEPS;
                term = RT_RAY_UNFINISHED + 16u;
            } else if (r < Bp->r_capture) {
                term = RT_RAY_CAPTURED;
            } else if (r > Bp->r_esc) {
                term = RT_RAY_ESCAPED;
            } else if (q.acc + q.rej >= Bp->max_steps) {
                q.flags |= RT_RAYFLAG_MAX_STEPS;
                term = RT_RAY_UNFINISHED + 16u;
            } else {
                const double cap = Bp->cap_c * fmax(r - Bp->rh, 0.01 * Bp->m);
                if (fabs(q.h) > cap) q.h = -cap;
                if (fabs(q.h) < 1e-8) {
                    q.flags |= RT_RAYFLAG_STEP_UNDERFLOW;
                    term = RT_RAY_CAPTURED;
                }
            }
            if (!term && (q.critical || r < Bp->fp64_radius || r >= kFp32MaxRadius)) {
                q.mode = MODE_PARK;  // into the FP64 zone: the near pass takes it
                continue;
            }
            if (term) {
                finish_ray(Bp, S, tid + s * BLOCK, term & 15u, q.flags, q.acc, q.rej, q.wind, 0.0, 0.0, NAN, 1.0,
                           args.out, q.y);
                q.mode = MODE_IDLE;
                continue;
            }
            act[s] = true;
        }
        if (!(act[0] || act[1])) continue;

        // ---- FP32 stages of both slots (an inactive slot computes on its last state) ----
        float2 x0[3], p0[3], incx[3], incp[3], ex[3], ep[3], g7[3], kp7[3], r7, hf7, s7;
        const float2 hf2 = make_float2(static_cast<float>(st[0].h), static_cast<float>(st[1].h));
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            x0[i] = make_float2(static_cast<float>(st[0].y[i]), static_cast<float>(st[1].y[i]));
            p0[i] = make_float2(static_cast<float>(st[0].y[3 + i]), static_cast<float>(st[1].y[3 + i]));
        }
        far_stages(x0, p0, dx1, kp1, hf2, Mf, af, a2f, incx, incp, ex, ep, g7, kp7, r7, hf7, s7);
        n_rhs += 6u * (static_cast<uint32_t>(act[0]) + static_cast<uint32_t>(act[1]));

        // ---- per slot: FP64 solution, error norm, accept / reject, events, projection ----
#pragma unroll
        for (int s = 0; s < kSlots; ++s) {
            if (!act[s]) continue;
            SlotState& q = st[s];
            const BundleDesc* Bp = args.bundles + q.bidx;
            const double hh = q.h;
            double y5[6];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                y5[i] = fma(hh, q.y[3 + i], q.y[i]) + static_cast<double>(lane_of(incx[i], s));
                y5[3 + i] = q.y[3 + i] + static_cast<double>(lane_of(incp[i], s));
            }
            // error norm (rk45_adaptive.hpp:254-261) in FP64 on the FP32 estimate
            double err;
            {
                double num = 0.0, den = 1.0;
                const double rtol = Bp->rtol, atol = Bp->atol;
#pragma unroll
                for (int i = 0; i < 6; ++i) {
                    const double e = fabs(static_cast<double>(i < 3 ? lane_of(ex[i], s) : lane_of(ep[i - 3], s)));
                    const double sc = rtol * fmax(fabs(q.y[i]), fabs(y5[i])) + atol;
                    if (e * den > num * sc) {
                        num = e;
                        den = sc;
                    }
                }
                err = num / den;
            }
            if (!(err <= 1e300)) err = 1e300;  // non-finite trial: reject with the largest cut
            ++n_att;
            if (err > 1.0) {
                // reject (rk45_adaptive.hpp:303-311)
                ++q.rej;
                const float le = __log2f(fmaxf(static_cast<float>(err), 1e-12f));
                const float factor = pi30_factor(le, q.has_hist ? q.lnp : le, 4.0f);
                q.lnp = le;
                q.has_hist = true;
                q.h = -fabs(q.h) * clampd(0.9 * static_cast<double>(factor), 0.1, 0.9);
                continue;
            }
            ++q.acc;
            ++n_acc;
            bool finite = true;
#pragma unroll
            for (int i = 0; i < 6; ++i) finite = finite && isfinite(y5[i]);
            if (!finite) {
                q.flags |= RT_RAYFLAG_NONFINITE;
                finish_ray(Bp, S, tid + s * BLOCK, RT_RAY_CAPTURED, q.flags, q.acc, q.rej, q.wind, 0.0, 0.0, NAN, 1.0,
                           args.out, q.y);
                q.mode = MODE_IDLE;
                continue;
            }
            float r5 = lane_of(r7, s), H5 = lane_of(hf7, s), S5 = lane_of(s7, s);
            float gx[3], kp[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                gx[i] = lane_of(g7[i], s);
                kp[i] = lane_of(kp7[i], s);
            }
            if ((Bp->flags & BF_DISK) && q.y[2] * y5[2] <= 0.0 && q.y[2] != y5[2]) {
                const double sl = q.y[2] / (q.y[2] - y5[2]);
                const double xe = q.y[0] + sl * (y5[0] - q.y[0]);
                const double ye = q.y[1] + sl * (y5[1] - q.y[1]);
                const double a = Bp->a;
                const double re = sqrt(fmax(xe * xe + ye * ye - a * a, 0.0));
                const double margin = 0.05 * re + 0.5 * Bp->m;
                if (re >= Bp->r_in - margin && re <= Bp->r_out + margin) {
                    double xr[15];
                    const double rr = far_disk_step(Bp, q.y, hh, xr);
                    n_rhs += 7u;
                    ++n_redo;
                    if (rr > 0.0) {
                        // a disk hit: park the root point (r_hit in the step slot) for the finish pass
                        S.lambda[tid + s * BLOCK] += xr[6] * hh;
                        q.wind += branch_winding(q.y[0], q.y[1], xr[0], xr[1]);
#pragma unroll
                        for (int i = 0; i < 6; ++i) q.y[i] = xr[i];
                        q.h = rr;
                        q.mode = MODE_FINISHQ;
                        continue;
                    }
                    // off the disk: the FP64 step stands in for the FP32 one
#pragma unroll
                    for (int i = 0; i < 6; ++i) y5[i] = xr[i];
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        gx[i] = static_cast<float>(xr[6 + i] - xr[3 + i]);
                        kp[i] = static_cast<float>(xr[9 + i]);
                    }
                    r5 = static_cast<float>(xr[12]);
                    H5 = static_cast<float>(xr[13]);
                    S5 = static_cast<float>(xr[14]);
                }
            }
            // capture / escape / certain capture inside this step: the terminal point is
            // interpolated to the threshold radius (FP64 Hermite on the FSAL end points)
            {
                double target = 0.0;
                uint32_t term = 0;
                if (r5 < Bp->r_capture) {
                    term = RT_RAY_CAPTURED;
                    target = Bp->r_capture;
                } else if (r5 > Bp->r_esc) {
                    term = RT_RAY_ESCAPED;
                    target = Bp->r_esc;
                } else if (q.can_early != 0 && r5 < Bp->r_early) {
                    const double M = Bp->m, a = Bp->a;
                    if (q.can_early < 0)  // Carter test, once per ray, when first inside r_early
                        q.can_early = shadow_distance(M, a, 0.0, Bp->rh, S.lz0[tid + s * BLOCK],
                                                      S.q0[tid + s * BLOCK]) > kEarlyCaptureMargin;
                    const double rd = r5, rr2 = rd * rd, z = y5[2];
                    const double k70 = y5[3] + gx[0], k71 = y5[4] + gx[1], k72 = y5[5] + gx[2];
                    const double drdl = (rr2 * rd * (y5[0] * k70 + y5[1] * k71) + rd * (rr2 + a * a) * z * k72) /
                                        (rr2 * rr2 + a * a * z * z);
                    if (q.can_early > 0 && drdl > 0.0) {
                        term = RT_RAY_CAPTURED;
                        q.flags |= RT_RAYFLAG_EARLY_CAPTURE;
                        target = Bp->r_early;
                    }
                }
                if (term) {
                    double xch[24];
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        xch[i] = q.y[i];
                        xch[3 + i] = q.y[3 + i];
                        xch[6 + i] = q.y[3 + i] + static_cast<double>(lane_of(dx1[i], s));
                        xch[9 + i] = static_cast<double>(lane_of(kp1[i], s));
                        xch[12 + i] = y5[i];
                        xch[15 + i] = y5[3 + i];
                        xch[18 + i] = y5[3 + i] + static_cast<double>(gx[i]);
                        xch[21 + i] = static_cast<double>(kp[i]);
                    }
                    finish_ray(Bp, S, tid + s * BLOCK, term, q.flags, q.acc, q.rej, q.wind, target, hh, NAN, 1.0,
                               args.out, xch);
                    q.mode = MODE_IDLE;
                    continue;
                }
            }
            // projection onto H = 0 (closest root, rk45_adaptive.hpp:126-134), in FP64 with the
            // FSAL stage's H and s; n = dx/dlambda at y5, k.n and |n|^2 from |k| = 1
            double alpha = 0.0;
            {
                const double hf5 = H5, s5 = S5;
                const double pp = y5[3] * y5[3] + y5[4] * y5[4] + y5[5] * y5[5];
                const double res = 0.5 * (pp - 1.0 - 2.0 * hf5 * s5 * s5);
                const int j = tid + s * BLOCK;
                S.dH[j] = fmax(S.dH[j], fabs(res));
                if (fabs(res) >= Bp->proj_tol) {
                    const double hs = hf5 * s5;
                    const double kn = (s5 - 1.0) - 2.0 * hs;
                    const double pn = pp - 2.0 * hs * (s5 - 1.0);
                    const double nn = pp - 4.0 * hs * (s5 - 1.0) + 4.0 * hs * hs;
                    const double qa = 0.5 * (nn - 2.0 * hf5 * kn * kn);
                    const double qb = pn - 2.0 * hs * kn;
                    const double disc = qb * qb - 4.0 * qa * res;
                    if (disc >= 0.0) {
                        const double qq = -0.5 * (qb + copysign(sqrt(disc), qb));
                        if (qq != 0.0) alpha = res / qq;
                    }
                }
            }
            const float af32 = static_cast<float>(alpha);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float n = lane_of(incp[i], s) + lane_of(p0[i], s) + gx[i];  // FP32 image of n_i
                y5[3 + i] += alpha * (y5[3 + i] + static_cast<double>(gx[i]));
                // next FSAL stage: k7 (taken before the projection) against the projected p
                set_lane(dx1[i], s, fmaf(-af32, n, gx[i]));
                set_lane(kp1[i], s, kp[i]);
            }
            q.wind += branch_winding(q.y[0], q.y[1], y5[0], y5[1]);
            S.lambda[tid + s * BLOCK] += hh;
#pragma unroll
            for (int i = 0; i < 6; ++i) q.y[i] = y5[i];
            q.r = r5;
            float factor = 5.0f;
            if (err != 0.0) {
                const float le = __log2f(fmaxf(static_cast<float>(err), 1e-12f));
                factor = pi30_factor(le, q.has_hist ? q.lnp : le, 5.0f);
                q.lnp = le;
                q.has_hist = true;
            }
            const double ah = fabs(q.h) * clampd(0.9 * static_cast<double>(factor), 0.2, 5.0);
            q.h = -clampd(ah, 1e-8, 1e13);
        }
    }

    unsigned long long w_att = n_att, w_acc = n_acc, w_rays = n_rays, w_rhs = n_rhs, w_redo = n_redo;
    for (int off = 16; off > 0; off >>= 1) {
        w_redo += __shfl_down_sync(FULL, w_redo, off);
        w_att += __shfl_down_sync(FULL, w_att, off);
        w_acc += __shfl_down_sync(FULL, w_acc, off);
        w_rays += __shfl_down_sync(FULL, w_rays, off);
        w_rhs += __shfl_down_sync(FULL, w_rhs, off);
    }
    if (lane == 0) {
        atomicAdd(args.stats + ST_RAYS, w_rays);
        atomicAdd(args.stats + ST_ATTEMPTS, w_att);
        atomicAdd(args.stats + ST_ACCEPTED, w_acc);
        atomicAdd(args.stats + ST_RHS, w_rhs);
        atomicAdd(args.stats + ST_FP64_ATTEMPTS, w_redo);  // disk-crossing steps taken again in FP64
    }
}

// The far-pass kernel for a block size (64 or 128) and warps per SM (12 or 8).
const void* far_pair_kernel_for(uint32_t block, int warps_per_sm) {
    if (warps_per_sm == 8)
        return (block == 64) ? reinterpret_cast<const void*>(&far_pair_kernel<64, 8>)
                             : reinterpret_cast<const void*>(&far_pair_kernel<128, 8>);
    return (block == 64) ? reinterpret_cast<const void*>(&far_pair_kernel<64, 12>)
                         : reinterpret_cast<const void*>(&far_pair_kernel<128, 12>);
}

}  // namespace relsim
