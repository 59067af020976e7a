// rt_trace.cu -- persistent backward null-geodesic tracer for sm_100a.
//
// One ray per lane.  Warps claim rays from a global work counter; when at
// least `refill_threshold` lanes of a warp are idle the warp claims that many
// consecutive rays with one atomic (ballot + popc rank), so lanes whose rays
// terminated are refilled instead of idling while the warp's longest ray runs.
//
// Per ray: Dormand-Prince 5(4) on the Kerr-Schild Hamiltonian state (x, p)
// with p_t = -1 (kerr_schild_null_integrator.hpp:72-114), PI30 control
// (step_controller.hpp:51-58; accept/reject scaling rk45_adaptive.hpp:294-310),
// FSAL reuse of the last stage, a step cap |h| <= c max(r - r_+, 0.01 M),
// projection onto H = 0 after each accepted step, and classification:
// captured (r < capture_scale r_+, software_compute_engine.hpp:1667-1671),
// escaped (r > escape radius, :1672-1675), disk (first z = 0 crossing on
// [r_in, r_out], root by Illinois regula falsi on the DP5 solution of a step
// fraction), with the Carter certain-capture early-out
// (carter_ray_classifier.hpp:146-150).  Terminal points are interpolated to
// the threshold radius (cubic Hermite on the step's FSAL end points).
//
// Layout: the hot state (y, k1, r, h, counters) lives in registers; cold
// per-lane state (affine parameter, invariants at the start, root bracket) in
// shared memory as structure of arrays.  Ray set-up, termination and the
// Carter test are out of line so the step loop stays small in the
// instruction cache; states cross that boundary through small local arrays.
// The disk root solve reuses the loop's stage code: a lane in ROOT mode runs
// its next DP5 evaluation at a fraction of the step instead of a full step.
//
// The mixed-precision mode runs as two passes (PASS_FAR, PASS_NEAR) instead:
// an FP32-stage kernel for the far zone and an FP64 kernel for the zone near
// the hole, rays moving between them through queues with their state parked
// in HBM, disk crossings solved on the step's dense output, and disk hits
// written by a finish kernel.  Splitting the code this way keeps each loop
// small in the instruction cache (the single mixed kernel, which holds both
// step forms, is instruction-fetch bound).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "rt_device.cuh"
#include "rt_internal.h"
#include "rt_ray.cuh"

namespace relsim {

namespace {

// Mixed-precision DP45 step for the far zone.  The state y and the result y5
// are FP64; the stages run in FP32 on the deviation from free streaming:
//   x_j = x + h c_j p + h sum_m a_jm dx_m,   dx_m = (p_m - p) - 2 H s k (at stage m)
//   p_j = p + h sum_m a_jm kp_m,             kp_m = dp/dlambda (at stage m)
// so the large h p term of every position increment stays FP64 and FP32 only
// carries the gravitational part.  y5 = y + h p (FP64) + h sum b_j dx_j (FP32).
// The error estimate uses sum_j e_j = 0: E_x = h sum e_j dx_j.  Outputs k7 in
// FP64 (FSAL), |E| per component, and the FP32 BL radius, H and s of the FSAL
// stage at y5 (the step's bookkeeping: step cap, termination, projection).
// When the step crosses z = 0 it also writes the dense-output term
// e = h sum_j D_j k_j; sum_j D_j = 0 makes its position part h sum_j D_j dx_j,
// so it too comes from the FP32 deviations.
__device__ __forceinline__ void mixed_stages(const double* __restrict__ y, const double* __restrict__ k1, double hh,
                                             double M, double a, double* __restrict__ y5, double* __restrict__ k7,
                                             double* __restrict__ est, float& r7, float& hf7, float& s7,
                                             double* __restrict__ dense_e) {
    const float h = static_cast<float>(hh);
    const float Mf = static_cast<float>(M), af = static_cast<float>(a);
    float x0[3], p0[3];
    float dx1[3], kp1[3], dx2[3], kp2[3], dx3[3], kp3[3], dx4[3], kp4[3], dx5[3], kp5[3], dx6[3], kp6[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        x0[i] = static_cast<float>(y[i]);
        p0[i] = static_cast<float>(y[3 + i]);
        dx1[i] = static_cast<float>(k1[i] - y[3 + i]);
        kp1[i] = static_cast<float>(k1[3 + i]);
    }
    constexpr float C2 = 1.0f / 5.0f, C3 = 3.0f / 10.0f, C4 = 4.0f / 5.0f, C5 = 8.0f / 9.0f;
    float in[6], g[6], hf, sv;
#define RT_STAGE(DXO, KPO, CC, SUMX, SUMP)                          \
    _Pragma("unroll") for (int i = 0; i < 3; ++i) {                 \
        const float dp = h * (SUMP);                                \
        in[i] = x0[i] + h * ((CC) * p0[i] + (SUMX));                \
        in[3 + i] = p0[i] + dp;                                     \
        g[i] = dp;                                                  \
    }                                                               \
    {                                                               \
        float dpv[3] = {g[0], g[1], g[2]};                          \
        ks_rhs<float, true>(in, Mf, af, g, hf, sv);                 \
        _Pragma("unroll") for (int i = 0; i < 3; ++i) {             \
            DXO[i] = dpv[i] + g[i];                                 \
            KPO[i] = g[3 + i];                                      \
        }                                                           \
    }
    RT_STAGE(dx2, kp2, C2, float(DP::A21) * dx1[i], float(DP::A21) * kp1[i])
    RT_STAGE(dx3, kp3, C3, float(DP::A31) * dx1[i] + float(DP::A32) * dx2[i],
             float(DP::A31) * kp1[i] + float(DP::A32) * kp2[i])
    RT_STAGE(dx4, kp4, C4, float(DP::A41) * dx1[i] + float(DP::A42) * dx2[i] + float(DP::A43) * dx3[i],
             float(DP::A41) * kp1[i] + float(DP::A42) * kp2[i] + float(DP::A43) * kp3[i])
    RT_STAGE(dx5, kp5, C5,
             float(DP::A51) * dx1[i] + float(DP::A52) * dx2[i] + float(DP::A53) * dx3[i] + float(DP::A54) * dx4[i],
             float(DP::A51) * kp1[i] + float(DP::A52) * kp2[i] + float(DP::A53) * kp3[i] + float(DP::A54) * kp4[i])
    RT_STAGE(dx6, kp6, 1.0f,
             float(DP::A61) * dx1[i] + float(DP::A62) * dx2[i] + float(DP::A63) * dx3[i] + float(DP::A64) * dx4[i] +
                 float(DP::A65) * dx5[i],
             float(DP::A61) * kp1[i] + float(DP::A62) * kp2[i] + float(DP::A63) * kp3[i] + float(DP::A64) * kp4[i] +
                 float(DP::A65) * kp5[i])
#undef RT_STAGE
    // 5th-order solution: FP64 accumulation of the FP32 increments
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float sx = float(DP::B1) * dx1[i] + float(DP::B3) * dx3[i] + float(DP::B4) * dx4[i] +
                         float(DP::B5) * dx5[i] + float(DP::B6) * dx6[i];
        const float sp = float(DP::B1) * kp1[i] + float(DP::B3) * kp3[i] + float(DP::B4) * kp4[i] +
                         float(DP::B5) * kp5[i] + float(DP::B6) * kp6[i];
        y5[i] = y[i] + hh * y[3 + i] + static_cast<double>(h * sx);
        y5[3 + i] = y[3 + i] + static_cast<double>(h * sp);
    }
    // stage 7 (FSAL) at y5
#pragma unroll
    for (int i = 0; i < 6; ++i) in[i] = static_cast<float>(y5[i]);
    r7 = ks_rhs<float, true>(in, Mf, af, g, hf, sv);
    hf7 = hf;
    s7 = sv;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float dx7 = static_cast<float>(y5[3 + i] - y[3 + i]) + g[i];
        const float ex = float(DP::E1) * dx1[i] + float(DP::E3) * dx3[i] + float(DP::E4) * dx4[i] +
                         float(DP::E5) * dx5[i] + float(DP::E6) * dx6[i] + float(DP::E7) * dx7;
        const float ep = float(DP::E1) * kp1[i] + float(DP::E3) * kp3[i] + float(DP::E4) * kp4[i] +
                         float(DP::E5) * kp5[i] + float(DP::E6) * kp6[i] + float(DP::E7) * g[3 + i];
        est[i] = static_cast<double>(fabsf(h * ex));
        est[3 + i] = static_cast<double>(fabsf(h * ep));
        k7[i] = y5[3 + i] + static_cast<double>(g[i]);
        k7[3 + i] = static_cast<double>(g[3 + i]);
    }
    if (y[2] * y5[2] <= 0.0) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float dx7 = static_cast<float>(y5[3 + i] - y[3 + i]) + g[i];
            const float sx = float(DP::D1) * dx1[i] + float(DP::D3) * dx3[i] + float(DP::D4) * dx4[i] +
                             float(DP::D5) * dx5[i] + float(DP::D6) * dx6[i] + float(DP::D7) * dx7;
            const float sp = float(DP::D1) * kp1[i] + float(DP::D3) * kp3[i] + float(DP::D4) * kp4[i] +
                             float(DP::D5) * kp5[i] + float(DP::D6) * kp6[i] + float(DP::D7) * g[3 + i];
            dense_e[i] = static_cast<double>(h * sx);
            dense_e[3 + i] = static_cast<double>(h * sp);
        }
    }
}

// Dormand-Prince tableau rows for the rolled FP64 step: row s gives the
// coefficients of k1..k(s+1) in the input of stage s + 2 (row 5 = b, the
// 5th-order solution); kDpE are the error weights of k1..k7.
__constant__ double kDpA[6][6] = {
    {DP::A21, 0, 0, 0, 0, 0},
    {DP::A31, DP::A32, 0, 0, 0, 0},
    {DP::A41, DP::A42, DP::A43, 0, 0, 0},
    {DP::A51, DP::A52, DP::A53, DP::A54, 0, 0},
    {DP::A61, DP::A62, DP::A63, DP::A64, DP::A65, 0},
    {DP::B1, 0.0, DP::B3, DP::B4, DP::B5, DP::B6}};
__constant__ double kDpE[7] = {DP::E1, 0.0, DP::E3, DP::E4, DP::E5, DP::E6, DP::E7};

// Stage derivatives k2..k7 of the rolled FP64 step, per thread in shared memory.
template <int BLOCK>
struct KStore {
    double k[6][6][BLOCK];
};

// FP64 stages 2..7 as one rolled loop around a single RHS (small in the
// instruction cache; used where FP64 steps are a minority, e.g. the near zone
// of the mixed mode).  Same arithmetic as the straight-line form.
template <int BLOCK>
__device__ __forceinline__ void fp64_stages_rolled(const double* __restrict__ y, const double* __restrict__ k1,
                                                   double hh, double M, double a, KStore<BLOCK>& K, int tid,
                                                   bool root, double* __restrict__ y5, double* __restrict__ k7,
                                                   double* __restrict__ est, double& r5, double& hf5, double& s5) {
#pragma unroll 1
    for (int st = 0; st < 6; ++st) {
        double in[6];
        // the stage sum unrolled over j (predicated on j <= st): the shared-memory loads
        // of a stage are independent and issue up front instead of one per FMA
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double acc = kDpA[st][0] * k1[i];
#pragma unroll
            for (int j = 1; j < 6; ++j)
                if (j <= st) acc += kDpA[st][j] * K.k[j - 1][i][tid];
            in[i] = y[i] + hh * acc;
        }
        if (st == 5) {
#pragma unroll
            for (int i = 0; i < 6; ++i) y5[i] = in[i];
            if (root) return;
        }
        double out[6], hf, sv;
        const double rr = ks_rhs<double>(in, M, a, out, hf, sv);
#pragma unroll
        for (int i = 0; i < 6; ++i) K.k[st][i][tid] = out[i];
        if (st == 5) {
#pragma unroll
            for (int i = 0; i < 6; ++i) k7[i] = out[i];
            r5 = rr;
            hf5 = hf;
            s5 = sv;
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double acc = kDpE[0] * k1[i];
#pragma unroll
        for (int j = 2; j < 7; ++j) acc += kDpE[j] * K.k[j - 1][i][tid];
        est[i] = fabs(hh) * fabs(acc);
    }
}

}  // namespace

// 384 / BLOCK resident CTAs per SM caps the kernel at 168 registers per thread
// (12 warps per SM).
//
// PASS selects the single-kernel tracer or one pass of the two-pass mixed
// tracer.  The far pass (FP32 stages only) parks a ray when it enters the FP64
// zone; the near pass (FP64 stages) parks it back when it leaves the zone
// again.  Both passes solve disk crossings on the step's dense output.  Parked
// rays resume from their saved state, so a ray's arithmetic does not depend on
// which rays share its warp.
// Every form runs 12 warps per SM (168 registers); the pass kernels spill a
// little there, which measured faster than 8 warps without spills.
template <int BLOCK, bool MIXED, bool ROLLED, int PASS = PASS_SINGLE, int CONT = 0>
__global__ void __launch_bounds__(BLOCK, 384 / BLOCK) trace_kernel_t(TraceArgs args) {
    __shared__ Cold<BLOCK> S;
    __shared__ KStore<ROLLED ? BLOCK : 1> K;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    constexpr bool FAR_PASS = (PASS == PASS_FAR);
    constexpr bool NEAR_PASS = (PASS == PASS_NEAR);
    static_assert(!FAR_PASS || MIXED, "the far pass runs the FP32 stages");
    static_assert(!NEAR_PASS || !MIXED, "the near pass runs FP64 stages");
    // rays of this launch: pixels (single kernel, first far pass) or queue entries
    // (later passes; the single kernel as the critical pass of a two-pass launch)
    const bool from_queue =
        (PASS == PASS_SINGLE) ? (args.in_queue != nullptr) : !(FAR_PASS && args.from_pixels != 0);
    const uint64_t total = from_queue ? static_cast<uint64_t>(*args.in_count) : args.total_rays;

    // hot lane state
    double y[6], k1[6];
    double r = 0.0, h = 0.0;
    float lnp = 0.0f;  // log2 of the previous error (PI30 history)
    uint32_t acc = 0, rej = 0, flags = 0, bidx = 0;
    int mode = MODE_IDLE, wind = 0, can_early = 0;
    bool has_hist = false;
    bool critical = false;  // mixed mode: a near-critical ray (FP64 from its first step)
    float tol_sc = 1.0f;    // tolerance factor of the ray (critical_tol_scale for near-critical rays)
    bool k1_fp32 = false;  // k1 came from an FP32 far-zone stage (mixed mode)
    uint32_t guard = 0;    // loop iterations spent on the current ray
    uint32_t n_cross = 0;  // disk crossings so far (translucent-disk continuation)
    uint64_t ray = 0;        // launch index of the lane's ray
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] = k1[i] = 0.0;

    // warp-uniform claim state: rays [chunk_next, chunk_end) belong to this warp
    bool queue_open = true;
    uint64_t chunk_next = 0, chunk_end = 0;
    uint32_t n_att = 0, n_acc = 0, n_rays = 0, n_rhs = 0, n_far = 0;

    for (;;) {
        if constexpr (PASS != PASS_SINGLE) {
            // park the lanes whose rays go to the other pass, and the disk hits for
            // the finish pass (one atomic per warp and queue)
            const unsigned pmask = __ballot_sync(FULL, mode == MODE_PARK);
            const unsigned fmask = __ballot_sync(FULL, mode == MODE_FINISHQ);
            if (pmask | fmask) {
                uint32_t pbase = 0, fbase = 0;
                if (pmask) {
                    const int leader = __ffs(pmask) - 1;
                    if (lane == leader) pbase = atomicAdd(args.out_count, static_cast<uint32_t>(__popc(pmask)));
                    pbase = __shfl_sync(FULL, pbase, leader);
                }
                if (fmask) {
                    const int leader = __ffs(fmask) - 1;
                    if (lane == leader) fbase = atomicAdd(args.finish_count, static_cast<uint32_t>(__popc(fmask)));
                    fbase = __shfl_sync(FULL, fbase, leader);
                }
                if (mode == MODE_PARK || mode == MODE_FINISHQ) {
                    if (mode == MODE_PARK)
                        args.out_queue[pbase + static_cast<uint32_t>(__popc(pmask & lt_mask))] = static_cast<uint32_t>(ray);
                    else
                        args.finish_queue[fbase + static_cast<uint32_t>(__popc(fmask & lt_mask))] =
                            static_cast<uint32_t>(ray);
                    double xch[7];
#pragma unroll
                    for (int i = 0; i < 6; ++i) xch[i] = y[i];
                    xch[6] = h;
                    const uint32_t misc = (has_hist ? PM_HAS_HIST : 0u) |
                                          (static_cast<uint32_t>(can_early + 1) << PM_EARLY_SHIFT) |
                                          (n_cross << PM_CROSS_SHIFT);
                    const uint32_t uch[PU_COUNT] = {acc, rej, flags, guard, static_cast<uint32_t>(wind), misc,
                                                    __float_as_uint(lnp)};
                    park_ray(args.park, ray, S, tid, xch, uch);
                    mode = MODE_IDLE;
                }
            }
            if constexpr (FAR_PASS) {
                // near-critical rays to the critical pass, before their first step
                const unsigned cmask = __ballot_sync(FULL, mode == MODE_CRITQ);
                if (cmask) {
                    const int leader = __ffs(cmask) - 1;
                    uint32_t cbase = 0;
                    if (lane == leader) cbase = atomicAdd(args.crit_count, static_cast<uint32_t>(__popc(cmask)));
                    cbase = __shfl_sync(FULL, cbase, leader);
                    if (mode == MODE_CRITQ) {
                        args.crit_queue[cbase + static_cast<uint32_t>(__popc(cmask & lt_mask))] =
                            static_cast<uint32_t>(ray);
                        mode = MODE_IDLE;
                    }
                }
            }
        }
        // ---- refill idle lanes: from the warp's chunk, then from a new chunk
        //      of `claim` consecutive rays (one global atomic per chunk) ----
        const unsigned idle = __ballot_sync(FULL, mode == MODE_IDLE);
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
                if (b >= total) {
                    queue_open = false;
                } else {
                    base2 = b;
                    got2 = true;
                    if (b + args.claim >= total) queue_open = false;
                }
            }
            const uint64_t used_old = (avail < static_cast<uint64_t>(n_idle)) ? avail : n_idle;
            if (mode == MODE_IDLE) {
                const uint64_t rank = static_cast<uint64_t>(__popc(idle & lt_mask));
                uint64_t rid = ~0ull;
                if (rank < avail) rid = chunk_next + rank;
                else if (got2) rid = base2 + (rank - avail);
                if (rid < total) {
                    uint64_t rix = rid;
                    if constexpr (PASS != PASS_SINGLE) {
                        rix = from_queue ? static_cast<uint64_t>(args.in_queue[rid]) : args.ray_base + rid;
                    } else {
                        if (from_queue) rix = args.in_queue[rid];
                    }
                    // bundle of this ray: last bundle whose ray_begin <= rix
                    uint32_t lo = 0, hi = args.n_bundles;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (args.bundles[mid].ray_begin <= rix) lo = mid; else hi = mid;
                    }
                    bidx = lo;
                    ray = rix;
                    bool resumed = false;
                    if constexpr (PASS != PASS_SINGLE) {
                        if (from_queue) {
                            double xch[13];
                            uint32_t uch[PU_COUNT];
                            r = resume_ray(args.bundles + lo, args.park, rix, rix - args.bundles[lo].ray_begin,
                                                  S, tid, xch, uch);
#pragma unroll
                            for (int i = 0; i < 6; ++i) {
                                y[i] = xch[i];
                                k1[i] = xch[6 + i];
                            }
                            h = xch[12];
                            acc = uch[PU_ACC];
                            rej = uch[PU_REJ];
                            flags = uch[PU_FLAGS];
                            guard = uch[PU_GUARD];
                            wind = static_cast<int>(uch[PU_WIND]);
                            has_hist = (uch[PU_MISC] & PM_HAS_HIST) != 0u;
                            can_early = static_cast<int>((uch[PU_MISC] >> PM_EARLY_SHIFT) & 3u) - 1;
                            if constexpr (CONT != 0) n_cross = (uch[PU_MISC] >> PM_CROSS_SHIFT) & 31u;
                            lnp = __uint_as_float(uch[PU_LNP]);
                            k1_fp32 = false;
                            mode = MODE_STEP;
                            ++n_rhs;
                            resumed = true;
                        }
                    }
                    if (!resumed) {
                        double xch[12];
                        const InitResult ir =
                            init_ray(args.bundles + lo, rix - args.bundles[lo].ray_begin, S, tid, xch);
#pragma unroll
                        for (int i = 0; i < 6; ++i) {
                            y[i] = xch[i];
                            k1[i] = xch[6 + i];
                        }
                        r = ir.r;
                        can_early = ir.can_early;
                        h = -args.bundles[lo].h0;
                        lnp = 0.0f;
                        has_hist = false;
                        acc = rej = flags = 0;
                        wind = args.bundles[lo].wind0;
                        k1_fp32 = false;
                        guard = 0;
                        n_cross = 0;
                        critical = false;
                        tol_sc = 1.0f;
                        const BundleDesc* Bc = args.bundles + lo;
                        // mixed mode: the distance of the ray's constants from the critical
                        // curve decides whether it is near-critical (and the Carter early
                        // capture, from the same value); the critical pass grades its
                        // tolerance with it
                        if ((MIXED && Bc->critical_band > 0.0f) || (PASS == PASS_SINGLE && !MIXED && from_queue)) {
                            const double db = shadow_distance(Bc->m, Bc->a, 0.0, Bc->rh, S.lz0[tid], S.q0[tid]);
                            if (can_early < 0) can_early = db > kEarlyCaptureMargin;
                            const double band = static_cast<double>(Bc->critical_band) * Bc->m;
                            critical = fabs(db) < band;
                            if (critical && PASS == PASS_SINGLE) tol_sc = critical_tol_scale(db, band);
                        }
                        mode = MODE_STEP;
                        if (!(PASS == PASS_SINGLE && from_queue)) ++n_rays;  // counted by the far pass
                        ++n_rhs;
                    }
                }
            }
            if (got2) {
                chunk_next = base2 + (static_cast<uint64_t>(n_idle) - used_old);
                chunk_end = base2 + args.claim;
                if (chunk_end > total) chunk_end = total;
            } else {
                chunk_next += used_old;
            }
        }
        if (__ballot_sync(FULL, mode != MODE_IDLE) == 0) {
            if (!queue_open && chunk_next >= chunk_end) break;
            continue;
        }
        // mixed mode: the warp takes an FP32 far-zone step only when no stepping
        // lane is inside the FP64 zone (one instruction stream per iteration;
        // lanes in a root solve always run FP64)
        bool far = false;
        if constexpr (FAR_PASS) {
            far = true;  // near-zone rays were parked for the near pass
        } else if constexpr (MIXED) {
            const bool stepping = (mode == MODE_STEP || mode == MODE_REDO);
            const BundleDesc* Bz = args.bundles + bidx;
            const bool lane_far = stepping && !critical && r >= Bz->fp64_radius && r < kFp32MaxRadius;
            // every lane executes the ballot (no short-circuit around a full-mask sync)
            const unsigned near_lanes = __ballot_sync(FULL, stepping && !lane_far);
            far = lane_far && near_lanes == 0u;
        }
        if (mode == MODE_IDLE) continue;

        const BundleDesc* Bp = args.bundles + bidx;
        const double M = Bp->m, a = Bp->a;
        // backstop: a ray needs at most 62 iterations per attempt (attempt, <= 60
        // root iterations, redo); past that bound it is ended as unfinished
        if (++guard > 64u * Bp->max_steps + 64u) {
            flags |= RT_RAYFLAG_MAX_STEPS;
            double xch[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) xch[i] = y[i];
            end_ray<(CONT != 0)>(args, Bp, S, tid, n_cross, RT_RAY_UNFINISHED, flags, acc, rej, wind, 0.0, 0.0, xch);
            mode = MODE_IDLE;
            continue;
        }
        double hh = h;
        if (mode == MODE_STEP) {
            // the initial point may already be outside the integration domain
            uint32_t term = 0;
            if (r < Bp->r_capture) term = RT_RAY_CAPTURED;
            else if (r > Bp->r_esc) term = RT_RAY_ESCAPED;
            else if (acc + rej >= Bp->max_steps) {
                flags |= RT_RAYFLAG_MAX_STEPS;
                term = RT_RAY_UNFINISHED + 16;
            }
            if (term == 0) {
                const double cap = Bp->cap_c * fmax(r - Bp->rh, 0.01 * M);
                if (fabs(h) > cap) h = -cap;
                hh = h;
                if (fabs(hh) < 1e-8) {
                    flags |= RT_RAYFLAG_STEP_UNDERFLOW;
                    term = RT_RAY_CAPTURED;
                }
            }
            if (term) {
                double xch[6];
#pragma unroll
                for (int i = 0; i < 6; ++i) xch[i] = y[i];
                end_ray<(CONT != 0)>(args, Bp, S, tid, n_cross, term & 15u, flags, acc, rej, wind, 0.0, 0.0, xch);
                mode = MODE_IDLE;
                continue;
            }
            if constexpr (FAR_PASS) {
                if (critical || r < Bp->fp64_radius || r >= kFp32MaxRadius) {  // into the FP64 zone
                    mode = critical ? MODE_CRITQ : MODE_PARK;
                    continue;
                }
            }
            if constexpr (NEAR_PASS) {
                if (args.allow_exit != 0u && r >= kNearExitFactor * Bp->fp64_radius &&
                    r < kFp32MaxRadius) {  // back out of the FP64 zone
                    mode = MODE_PARK;
                    continue;
                }
            }
        } else if (mode == MODE_ROOT) {
            const double lo = S.lo[tid], hi = S.hi[tid], flo = S.flo[tid], fhi = S.fhi[tid];
            double t = (lo * fhi - hi * flo) / (fhi - flo);
            if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
            S.troot[tid] = t;
            hh = t * h;
        }

        // ---- Dormand-Prince stages 2..7 (rk45_adaptive.hpp:210-252); stage 7 is
        //      the FSAL stage at the 5th-order solution y5.  kA holds k2 for
        //      stages 3..6, then k7; est holds |h| |sum_j e_j k_j| per component. ----
        double dense5[6];  // h sum_j D_j k_j of a step that crosses z = 0 (two-pass tracer)
        double kA[6], y5[6], est[6];
        double r5 = 0.0, hf5 = 0.0, s5 = 0.0;
        const bool root = (mode == MODE_ROOT);
        if (far) {
            // FP32 radius, H and s of the FSAL stage: the projection then holds
            // H = 0 to the FP32 stages' own accuracy
            float r7, hf7, s7;
            mixed_stages(y, k1, hh, M, a, y5, kA, est, r7, hf7, s7, dense5);
            r5 = r7;
            hf5 = hf7;
            s5 = s7;
            if (mode == MODE_STEP) ++n_far;
        } else if constexpr (!FAR_PASS) {
            if constexpr (MIXED) {
                if (k1_fp32) {  // entering the FP64 zone: first stage again in FP64
                    double hf, sv;
                    ks_rhs<double>(y, M, a, k1, hf, sv);
                    k1_fp32 = false;
                    ++n_rhs;
                }
            }
            if constexpr (ROLLED) {
                fp64_stages_rolled<BLOCK>(y, k1, hh, M, a, K, tid, root, y5, kA, est, r5, hf5, s5);
                if constexpr (NEAR_PASS) {
                    if (y[2] * y5[2] <= 0.0) {  // dense-output term; K holds k2..k7
#pragma unroll
                        for (int i = 0; i < 6; ++i)
                            dense5[i] = hh * (DP::D1 * k1[i] + DP::D3 * K.k[1][i][tid] + DP::D4 * K.k[2][i][tid] +
                                              DP::D5 * K.k[3][i][tid] + DP::D6 * K.k[4][i][tid] + DP::D7 * kA[i]);
                    }
                }
            } else {
                double k3[6], k4[6], k5[6], k6[6];
                double in[6], hf, sv;
#pragma unroll
                for (int i = 0; i < 6; ++i) in[i] = y[i] + hh * (DP::A21 * k1[i]);
                ks_rhs<double>(in, M, a, kA, hf, sv);
#pragma unroll
                for (int i = 0; i < 6; ++i) in[i] = y[i] + hh * (DP::A31 * k1[i] + DP::A32 * kA[i]);
                ks_rhs<double>(in, M, a, k3, hf, sv);
#pragma unroll
                for (int i = 0; i < 6; ++i)
                    in[i] = y[i] + hh * (DP::A41 * k1[i] + DP::A42 * kA[i] + DP::A43 * k3[i]);
                ks_rhs<double>(in, M, a, k4, hf, sv);
#pragma unroll
                for (int i = 0; i < 6; ++i)
                    in[i] = y[i] + hh * (DP::A51 * k1[i] + DP::A52 * kA[i] + DP::A53 * k3[i] + DP::A54 * k4[i]);
                ks_rhs<double>(in, M, a, k5, hf, sv);
#pragma unroll
                for (int i = 0; i < 6; ++i)
                    in[i] = y[i] + hh * (DP::A61 * k1[i] + DP::A62 * kA[i] + DP::A63 * k3[i] + DP::A64 * k4[i] +
                                         DP::A65 * k5[i]);
                ks_rhs<double>(in, M, a, k6, hf, sv);
#pragma unroll
                for (int i = 0; i < 6; ++i)
                    y5[i] = y[i] + hh * (DP::B1 * k1[i] + DP::B3 * k3[i] + DP::B4 * k4[i] + DP::B5 * k5[i] +
                                         DP::B6 * k6[i]);
                if (!root) {
                    r5 = ks_rhs<double>(y5, M, a, kA, hf5, s5);
#pragma unroll
                    for (int i = 0; i < 6; ++i)
                        est[i] = fabs(hh) * fabs(DP::E1 * k1[i] + DP::E3 * k3[i] + DP::E4 * k4[i] +
                                                 DP::E5 * k5[i] + DP::E6 * k6[i] + DP::E7 * kA[i]);
                    if constexpr (NEAR_PASS) {
                        if (y[2] * y5[2] <= 0.0) {
#pragma unroll
                            for (int i = 0; i < 6; ++i)
                                dense5[i] = hh * (DP::D1 * k1[i] + DP::D3 * k3[i] + DP::D4 * k4[i] +
                                                  DP::D5 * k5[i] + DP::D6 * k6[i] + DP::D7 * kA[i]);
                        }
                    }
                }
            }
        }
        n_rhs += root ? 5 : 6;

        if (PASS == PASS_SINGLE && root) {
            const double ft = y5[2];
            const int rit = ++S.rit[tid];
            const double lo = S.lo[tid], hi = S.hi[tid];
            const bool done = (ft == 0.0) || (fabs(hi - lo) < 1e-15) ||
                              (fabs(ft) < 1e-13 * (1.0 + fabs(y5[0]) + fabs(y5[1]))) || (rit >= 60);
            if (done) {
                const double rr = sqrt(bl_r2<double>(y5[0], y5[1], y5[2], a * a));
                if (rr >= Bp->r_in && rr <= Bp->r_out && rr > Bp->rh * 1.02) {
                    // lambda at the root, one rounding in every kernel variant
                    const double lambda_step = S.lambda[tid];
                    S.lambda[tid] = fma(S.troot[tid], h, lambda_step);
                    double xch[18];
#pragma unroll
                    for (int i = 0; i < 6; ++i) {
                        xch[i] = y[i];
                        xch[12 + i] = y5[i];
                    }
                    if (n_cross == 0)
                        finish_ray(Bp, S, tid, RT_RAY_DISK, flags, acc, rej, wind, 0.0, 0.0, rr,
                                   disk_redshift(M, a, rr, S.lz0[tid]), args.out, xch);
                    mode = MODE_IDLE;
                    if constexpr (CONT != 0) {
                        // translucent disk: record the crossing and go on through it
                        record_crossing(args, Bp, S, tid, n_cross, y5,
                                        wind + branch_winding(y[0], y[1], y5[0], y5[1]));
                        ++n_cross;
                        if (n_cross < kMaxCrossings) {
                            S.lambda[tid] = lambda_step;
                            mode = MODE_REDO;  // the full step again, accepted as it stands
                        } else {
                            end_continuation(args, Bp, S, tid, n_cross, RT_RAY_UNFINISHED, y5);
                        }
                    }
                } else {
                    mode = MODE_REDO;  // not on the disk: take the full step again
                }
            } else {
                const double t = S.troot[tid];
                const int side = S.side[tid];
                if ((ft > 0.0) == (S.fhi[tid] > 0.0)) {
                    S.hi[tid] = t;
                    S.fhi[tid] = ft;
                    if (side == -1) S.flo[tid] *= 0.5;
                    S.side[tid] = -1;
                } else {
                    S.lo[tid] = t;
                    S.flo[tid] = ft;
                    if (side == 1) S.fhi[tid] *= 0.5;
                    S.side[tid] = 1;
                }
            }
            continue;
        }

        // error norm (rk45_adaptive.hpp:254-261) in FP64 in every mode (in the
        // far pass on the FP32 stages' estimate); kA holds k7
        double err;
        {
            double num = 0.0, den = 1.0;
            const double rtol = Bp->rtol * static_cast<double>(tol_sc), atol = Bp->atol * static_cast<double>(tol_sc);
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const double sc = rtol * fmax(fabs(y[i]), fabs(y5[i])) + atol;
                if (est[i] * den > num * sc) {
                    num = est[i];
                    den = sc;
                }
            }
            err = num / den;
        }
        if (!(err <= 1e300)) err = 1e300;  // non-finite trial: reject with the largest cut

        if (mode == MODE_STEP) {
            ++n_att;
            if (err > 1.0) {
                // reject (rk45_adaptive.hpp:303-311)
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
                flags |= RT_RAYFLAG_NONFINITE;
                double xch[6];
#pragma unroll
                for (int i = 0; i < 6; ++i) xch[i] = y[i];
                end_ray<(CONT != 0)>(args, Bp, S, tid, n_cross, RT_RAY_CAPTURED, flags, acc, rej, wind, 0.0, 0.0, xch);
                mode = MODE_IDLE;
                continue;
            }
            if ((Bp->flags & BF_DISK) && y[2] * y5[2] <= 0.0 && y[2] != y5[2]) {
                const double sl = y[2] / (y[2] - y5[2]);
                const double xe = y[0] + sl * (y5[0] - y[0]);
                const double ye = y[1] + sl * (y5[1] - y[1]);
                const double re = sqrt(fmax(xe * xe + ye * ye - a * a, 0.0));
                const double margin = 0.05 * re + 0.5 * M;
                if (re >= Bp->r_in - margin && re <= Bp->r_out + margin) {
                    if constexpr (PASS != PASS_SINGLE) {
                        // FP64 root on the step's dense output (its correction term from
                        // this step's stages: FP32 in the far pass, FP64 in the near
                        // pass); off the disk the step is accepted as it is
                        double xr[18];
                        const double t = dense_disk_root(y, k1, y5, kA, dense5, hh, xr + 12);
                        const double rr = sqrt(bl_r2<double>(xr[12], xr[13], xr[14], a * a));
                        if (rr >= Bp->r_in && rr <= Bp->r_out && rr > Bp->rh * 1.02) {
                            const int wroot = wind + branch_winding(y[0], y[1], xr[12], xr[13]);
                            if constexpr (!CONT) {
                                // a disk hit: park the root point (r_hit in the step slot) for
                                // the finish pass, which writes the record in lockstep
                                S.lambda[tid] = fma(t, hh, S.lambda[tid]);
                                wind = wroot;
#pragma unroll
                                for (int i = 0; i < 6; ++i) y[i] = xr[12 + i];
                                h = rr;
                                mode = MODE_FINISHQ;
                                continue;
                            }
                            // translucent disk: the first hit's record now, the crossing
                            // recorded, and the step accepted as it stands
                            if (n_cross == 0) {
                                // finish_ray takes the root point in xr[0..5] and xr[12..17]
#pragma unroll
                                for (int i = 0; i < 6; ++i) xr[i] = xr[12 + i];
                                const double lambda_step = S.lambda[tid];
                                S.lambda[tid] = fma(t, hh, lambda_step);
                                finish_ray(Bp, S, tid, RT_RAY_DISK, flags, acc, rej, wroot, 0.0, 0.0, rr,
                                           disk_redshift(M, a, rr, S.lz0[tid]), args.out, xr);
                                S.lambda[tid] = lambda_step;
                            }
                            record_crossing(args, Bp, S, tid, n_cross, xr + 12, wroot);
                            ++n_cross;
                            if (n_cross >= kMaxCrossings) {
                                end_continuation(args, Bp, S, tid, n_cross, RT_RAY_UNFINISHED, xr + 12);
                                mode = MODE_IDLE;
                                continue;
                            }
                        }
                    } else {
                        mode = MODE_ROOT;
                        S.lo[tid] = 0.0;
                        S.flo[tid] = y[2];
                        S.hi[tid] = 1.0;
                        S.fhi[tid] = y5[2];
                        S.side[tid] = 0;
                        S.rit[tid] = 0;
                        continue;
                    }
                }
            }
        }
        // accept, second half (also the REDO of a crossing off the disk)
        mode = MODE_STEP;
        {
            // capture / escape / certain capture inside this step: the terminal point is
            // interpolated to the threshold radius, independent of where the step ended
            double target = 0.0;
            uint32_t term = 0;
            if (r5 < Bp->r_capture) {
                term = RT_RAY_CAPTURED;
                target = Bp->r_capture;
            } else if (r5 > Bp->r_esc) {
                term = RT_RAY_ESCAPED;
                target = Bp->r_esc;
            } else if (can_early != 0 && r5 < Bp->r_early) {
                if (can_early < 0)  // Carter test, once per ray, when first inside r_early
                    can_early = shadow_distance(M, a, 0.0, Bp->rh, S.lz0[tid], S.q0[tid]) > kEarlyCaptureMargin;
                // dr_BL/dlambda (kerr_invariants.hpp:140); the trace runs towards
                // decreasing lambda, so dr/dlambda > 0 means inwards
                const double rr2 = r5 * r5, z = y5[2];
                const double drdl = (rr2 * r5 * (y5[0] * kA[0] + y5[1] * kA[1]) + r5 * (rr2 + a * a) * z * kA[2]) /
                                    (rr2 * rr2 + a * a * z * z);
                if (can_early > 0 && drdl > 0.0) {
                    term = RT_RAY_CAPTURED;
                    flags |= RT_RAYFLAG_EARLY_CAPTURE;
                    target = Bp->r_early;
                }
            }
            if (term) {
                double xch[24];
#pragma unroll
                for (int i = 0; i < 6; ++i) {
                    xch[i] = y[i];
                    xch[6 + i] = k1[i];
                    xch[12 + i] = y5[i];
                    xch[18 + i] = kA[i];
                }
                end_ray<(CONT != 0)>(args, Bp, S, tid, n_cross, term, flags, acc, rej, wind, target, hh, xch);
                mode = MODE_IDLE;
                continue;
            }
        }
        {
            // projection onto H = 0 (closest root, rk45_adaptive.hpp:126-134); n = dx/dl = k7[0..2],
            // k.n and |n|^2 from |k| = 1
            double* p = y5 + 3;
            const double pp = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
            const double res = 0.5 * (pp - 1.0 - 2.0 * hf5 * s5 * s5);
            S.dH[tid] = fmax(S.dH[tid], fabs(res));
            if (fabs(res) >= Bp->proj_tol) {
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
                        p[0] += alpha * kA[0];
                        p[1] += alpha * kA[1];
                        p[2] += alpha * kA[2];
                    }
                }
            }
        }
        if constexpr (CONT == 2) {
            // hydro model 2: the step's chord through the Fishbone-Moncrief torus
            // (software_compute_engine.hpp:1725-1731)
            double from[3], to[3];
            bl_cartesian(y, a, from);
            bl_cartesian(y5, a, to);
            fm_segment(*args.cont.shade, from, to, S.lz0[tid],
                       args.cont.vol + (Bp->out_offset + S.local[tid]) * VL_COUNT);
        }
        wind += branch_winding(y[0], y[1], y5[0], y5[1]);
        S.lambda[tid] += hh;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            y[i] = y5[i];
            k1[i] = kA[i];
        }
        r = r5;
        if constexpr (MIXED) k1_fp32 = far;
        float factor = 5.0f;
        if (err != 0.0) {
            const float le = __log2f(fmaxf(static_cast<float>(err), 1e-12f));
            factor = pi30_factor(le, has_hist ? lnp : le, 5.0f);
            lnp = le;
            has_hist = true;
        }
        const double ah = fabs(h) * clampd(0.9 * static_cast<double>(factor), 0.2, 5.0);
        h = -clampd(ah, 1e-8, 1e13);
    }

    // warp-reduced counters (per-lane counts fit 32 bits; the sums are 64-bit)
    unsigned long long w_att = n_att, w_acc = n_acc, w_rays = n_rays, w_rhs = n_rhs, w_far = n_far;
    for (int off = 16; off > 0; off >>= 1) {
        w_att += __shfl_down_sync(FULL, w_att, off);
        w_acc += __shfl_down_sync(FULL, w_acc, off);
        w_rays += __shfl_down_sync(FULL, w_rays, off);
        w_rhs += __shfl_down_sync(FULL, w_rhs, off);
        w_far += __shfl_down_sync(FULL, w_far, off);
    }
    if (lane == 0) {
        atomicAdd(args.stats + ST_RAYS, w_rays);
        atomicAdd(args.stats + ST_ATTEMPTS, w_att);
        atomicAdd(args.stats + ST_ACCEPTED, w_acc);
        atomicAdd(args.stats + ST_RHS, w_rhs);
        atomicAdd(args.stats + ST_FP64_ATTEMPTS, w_att - w_far);
    }
}

// unshaded launches (CONT = 0), shaded ones that follow rays through the
// translucent disk (CONT = 1) and, for hydro model 2, the FP64 tracer that
// gathers the Fishbone-Moncrief torus's light step by step (CONT = 2)
template __global__ void trace_kernel_t<64, false, false>(TraceArgs);
template __global__ void trace_kernel_t<128, false, false>(TraceArgs);
template __global__ void trace_kernel_t<256, false, false>(TraceArgs);
template __global__ void trace_kernel_t<64, false, true>(TraceArgs);
template __global__ void trace_kernel_t<128, false, true>(TraceArgs);
template __global__ void trace_kernel_t<64, true, true>(TraceArgs);
template __global__ void trace_kernel_t<128, true, true>(TraceArgs);
template __global__ void trace_kernel_t<64, true, false, PASS_FAR>(TraceArgs);
template __global__ void trace_kernel_t<128, true, false, PASS_FAR>(TraceArgs);
template __global__ void trace_kernel_t<64, false, false, PASS_NEAR>(TraceArgs);
template __global__ void trace_kernel_t<128, false, false, PASS_NEAR>(TraceArgs);
template __global__ void trace_kernel_t<64, false, false, PASS_SINGLE, 1>(TraceArgs);
template __global__ void trace_kernel_t<128, false, false, PASS_SINGLE, 1>(TraceArgs);
template __global__ void trace_kernel_t<256, false, false, PASS_SINGLE, 1>(TraceArgs);
template __global__ void trace_kernel_t<64, false, true, PASS_SINGLE, 1>(TraceArgs);
template __global__ void trace_kernel_t<128, false, true, PASS_SINGLE, 1>(TraceArgs);
template __global__ void trace_kernel_t<64, true, true, PASS_SINGLE, 1>(TraceArgs);
template __global__ void trace_kernel_t<128, true, true, PASS_SINGLE, 1>(TraceArgs);
template __global__ void trace_kernel_t<128, false, false, PASS_SINGLE, 2>(TraceArgs);
template __global__ void trace_kernel_t<64, true, false, PASS_FAR, true>(TraceArgs);
template __global__ void trace_kernel_t<128, true, false, PASS_FAR, true>(TraceArgs);
template __global__ void trace_kernel_t<64, false, false, PASS_NEAR, true>(TraceArgs);
template __global__ void trace_kernel_t<128, false, false, PASS_NEAR, true>(TraceArgs);

namespace {
// Mixed precision always uses the rolled FP64 step (its FP64 steps are a
// minority; the rolled form keeps the loop small).  Rolled kernels exist for
// 64- and 128-thread blocks (their stage store is 36 KB of shared memory at 128).
template <int CONT>
const void* kernel_for_t(uint32_t block, bool mixed, bool rolled) {
    if (mixed) {
        return (block == 64) ? reinterpret_cast<const void*>(&trace_kernel_t<64, true, true, PASS_SINGLE, CONT>)
                             : reinterpret_cast<const void*>(&trace_kernel_t<128, true, true, PASS_SINGLE, CONT>);
    }
    if (rolled) {
        return (block == 64) ? reinterpret_cast<const void*>(&trace_kernel_t<64, false, true, PASS_SINGLE, CONT>)
                             : reinterpret_cast<const void*>(&trace_kernel_t<128, false, true, PASS_SINGLE, CONT>);
    }
    switch (block) {
        case 64: return reinterpret_cast<const void*>(&trace_kernel_t<64, false, false, PASS_SINGLE, CONT>);
        case 256: return reinterpret_cast<const void*>(&trace_kernel_t<256, false, false, PASS_SINGLE, CONT>);
        default: return reinterpret_cast<const void*>(&trace_kernel_t<128, false, false, PASS_SINGLE, CONT>);
    }
}

const void* kernel_for(uint32_t block, bool mixed, bool rolled, int cont = 0) {
    if (cont == 2) return reinterpret_cast<const void*>(&trace_kernel_t<128, false, false, PASS_SINGLE, 2>);
    return (cont == 1) ? kernel_for_t<1>(block, mixed, rolled) : kernel_for_t<0>(block, mixed, rolled);
}
}  // namespace

uint32_t kernel_block(uint32_t block, bool mixed, bool rolled) {
    if ((mixed || rolled) && block > 128) return 128;
    return block;
}

int trace_occupancy(uint32_t block, bool mixed, bool rolled) {
    int n = 0;
    block = kernel_block(block, mixed, rolled);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_for(block, mixed, rolled), static_cast<int>(block), 0) !=
        cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n;
}

// Finish pass of the two-pass mixed tracer: the record and pixel of every disk
// hit parked by the far and near passes (root point, r_hit in the step slot).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) finish_kernel_t(TraceArgs args) {
    __shared__ Cold<BLOCK> S;
    const int tid = threadIdx.x;
    const uint64_t count = *args.in_count;
    const uint64_t n = args.park.n;
    for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * BLOCK + tid; j < count;
         j += static_cast<uint64_t>(gridDim.x) * BLOCK) {
        const uint64_t ray = args.in_queue[j];
        uint32_t lo = 0, hi = args.n_bundles;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (args.bundles[mid].ray_begin <= ray) lo = mid; else hi = mid;
        }
        const BundleDesc* Bp = args.bundles + lo;
        double xch[18];
#pragma unroll
        for (int i = 0; i < 6; ++i) xch[i] = xch[12 + i] = args.park.d[(PD_Y + i) * n + ray];
        const double r_hit = args.park.d[PD_H * n + ray];
        S.lambda[tid] = args.park.d[PD_LAMBDA * n + ray];
        S.dH[tid] = args.park.d[PD_DH * n + ray];
        S.lz0[tid] = args.park.d[PD_LZ0 * n + ray];
        S.q0[tid] = args.park.d[PD_Q0 * n + ray];
        S.local[tid] = ray - Bp->ray_begin;
        finish_ray(Bp, S, tid, RT_RAY_DISK, args.park.u[PU_FLAGS * n + ray], args.park.u[PU_ACC * n + ray],
                          args.park.u[PU_REJ * n + ray], static_cast<int>(args.park.u[PU_WIND * n + ray]), 0.0, 0.0,
                          r_hit, disk_redshift(Bp->m, Bp->a, r_hit, S.lz0[tid]), args.out, xch);
    }
}
template __global__ void finish_kernel_t<128>(TraceArgs);

namespace {
template <bool CONT>
const void* pass_kernel_t(int pass, uint32_t block) {
    if (pass == PASS_FAR)
        return (block == 64) ? reinterpret_cast<const void*>(&trace_kernel_t<64, true, false, PASS_FAR, CONT>)
                             : reinterpret_cast<const void*>(&trace_kernel_t<128, true, false, PASS_FAR, CONT>);
    return (block == 64) ? reinterpret_cast<const void*>(&trace_kernel_t<64, false, false, PASS_NEAR, CONT>)
                         : reinterpret_cast<const void*>(&trace_kernel_t<128, false, false, PASS_NEAR, CONT>);
}

const void* pass_kernel(int pass, uint32_t block, bool cont = false) {
    return cont ? pass_kernel_t<true>(pass, block) : pass_kernel_t<false>(pass, block);
}
}  // namespace

int trace_pass_occupancy(int pass, uint32_t block) {
    int n = 0;
    block = (block == 64) ? 64u : 128u;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pass_kernel(pass, block), static_cast<int>(block), 0) !=
        cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n;
}

void launch_trace_pass(const TraceArgs& args, int pass, uint32_t grid, uint32_t block, void* stream) {
    void* params[] = {const_cast<TraceArgs*>(&args)};
    block = (block == 64) ? 64u : 128u;
    cudaLaunchKernel(pass_kernel(pass, block, args.cont.cross != nullptr), dim3(grid), dim3(block), params, 0,
                     static_cast<cudaStream_t>(stream));
}

// Rounds of the two-pass mixed tracer: far pass (FP32) then near pass (FP64),
// the last near pass keeping every ray to its end.  A ray typically needs one
// round (in to a disk crossing or the near zone, and out); rays left after the
// last far pass finish in FP64.
constexpr int kMixedRounds = 4;
// Refill threshold of the near pass: its rays resume from parked state (a few
// loads and one RHS), so refilling a partly idle warp is cheap, while the
// near-zone work per ray (disk root, photon-region orbits) varies widely.
constexpr uint32_t kNearRefill = 16;  // measured best of 1, 4, 8, 16, 32
// Block of the critical pass (the FP64 kernel's default shape).
constexpr uint32_t kCriticalBlock = 128;

uint64_t two_pass_state_bytes(uint64_t n) {
    return n * (sizeof(double) * PD_COUNT + sizeof(uint32_t) * PU_COUNT + 4 * sizeof(uint32_t));
}

// Per-band queue counters (kBandCounterBytes): [0] far-pass claim (u64), [8]
// near queue count (u32), [12] far queue count (u32), [16] near-pass claim
// (u64), zeroed pairwise before each pass; [24] finish queue count (u32), [32]
// near-critical queue count (u32) and [40] the critical pass's claim (u64),
// zeroed once.
namespace {
cudaError_t enqueue_band(TraceArgs args, const TwoPassBuffers& buf, uint64_t begin, uint64_t count, char* qb,
                         uint32_t far_grid, uint32_t far_block, uint32_t near_grid, uint32_t finish_grid,
                         uint32_t crit_grid, bool crit_beside, cudaStream_t s) {
    uint32_t* near_q = buf.queues + 4 * begin;
    uint32_t* far_q = near_q + count;
    uint32_t* crit_q = far_q + 2 * count;
    args.park = buf.park;
    args.total_rays = count;
    args.ray_base = begin;
    args.finish_queue = far_q + count;
    args.finish_count = reinterpret_cast<uint32_t*>(qb + 24);
    const uint32_t far_refill = args.refill_threshold;
    cudaError_t e = cudaMemsetAsync(qb + 24, 0, 24, s);
    for (int round = 0; e == cudaSuccess && round < kMixedRounds; ++round) {
        // far pass: pixels (first round) or the far queue -> near queue
        if ((e = cudaMemsetAsync(qb, 0, 12, s)) != cudaSuccess) break;
        args.queue = reinterpret_cast<unsigned long long*>(qb);
        args.refill_threshold = far_refill;
        args.from_pixels = (round == 0) ? 1u : 0u;
        args.allow_exit = 0;
        args.in_queue = far_q;
        args.in_count = reinterpret_cast<const uint32_t*>(qb + 12);
        args.out_queue = near_q;
        args.out_count = reinterpret_cast<uint32_t*>(qb + 8);
        args.crit_queue = (round == 0) ? crit_q : nullptr;
        args.crit_count = (round == 0) ? reinterpret_cast<uint32_t*>(qb + 32) : nullptr;
        launch_trace_pass(args, PASS_FAR, far_grid, far_block, s);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        if (round == 0) {
            // critical pass: the near-critical rays, FP64 from their pixels to their
            // end at their graded tolerance (the single FP64 kernel over a queue);
            // on its own stream it runs beside the near passes, each filling the
            // SMs the other's tail leaves idle
            TraceArgs c = args;
            c.queue = reinterpret_cast<unsigned long long*>(qb + 40);
            c.refill_threshold = 32;
            c.in_queue = crit_q;
            c.in_count = reinterpret_cast<const uint32_t*>(qb + 32);
            c.out_queue = c.finish_queue = c.crit_queue = nullptr;
            c.out_count = c.finish_count = c.crit_count = nullptr;
            cudaStream_t cs = s;
            if (crit_beside) {
                cs = static_cast<cudaStream_t>(buf.crit_stream);
                if ((e = cudaEventRecord(static_cast<cudaEvent_t>(buf.crit_fork), s)) != cudaSuccess) break;
                if ((e = cudaStreamWaitEvent(cs, static_cast<cudaEvent_t>(buf.crit_fork), 0)) != cudaSuccess) break;
            }
            launch_trace(c, crit_grid, kCriticalBlock, false, false, cs);
            if ((e = cudaGetLastError()) != cudaSuccess) break;
            if (crit_beside && (e = cudaEventRecord(static_cast<cudaEvent_t>(buf.crit_join), cs)) != cudaSuccess) break;
        }
        // near pass: near queue -> far queue (the last one keeps its rays)
        if ((e = cudaMemsetAsync(qb + 12, 0, 12, s)) != cudaSuccess) break;
        args.queue = reinterpret_cast<unsigned long long*>(qb + 16);
        args.refill_threshold = far_refill < kNearRefill ? far_refill : kNearRefill;
        args.from_pixels = 0;
        args.allow_exit = (round + 1 < kMixedRounds) ? 1u : 0u;
        args.in_queue = near_q;
        args.in_count = reinterpret_cast<const uint32_t*>(qb + 8);
        args.out_queue = far_q;
        args.out_count = reinterpret_cast<uint32_t*>(qb + 12);
        launch_trace_pass(args, PASS_NEAR, near_grid, 128, s);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    // finish pass over the band's parked disk hits
    args.in_queue = args.finish_queue;
    args.in_count = args.finish_count;
    finish_kernel_t<128><<<finish_grid, 128, 0, s>>>(args);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (crit_beside) e = cudaStreamWaitEvent(s, static_cast<cudaEvent_t>(buf.crit_join), 0);
    return e;
}
}  // namespace

int enqueue_two_pass(const TraceArgs& base, const TwoPassBuffers& buf, int sm_count, uint32_t far_block,
                     void* stream, void* stream2, void* fork, void* join, uint32_t bands, BandHook after_band,
                     void* hook_ctx) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStream_t s2 = static_cast<cudaStream_t>(stream2);
    const uint64_t n = base.total_rays;
    if (!s2 || !fork || !join) bands = 1;
    bands = bands < 1 ? 1 : (bands > kMaxBands ? kMaxBands : bands);
    if (static_cast<uint64_t>(bands) > n) bands = static_cast<uint32_t>(n > 0 ? n : 1);
    far_block = (far_block == 64) ? 64u : 128u;
    const int far_occ = trace_pass_occupancy(PASS_FAR, far_block);
    const int near_occ = trace_pass_occupancy(PASS_NEAR, 128);
    const uint32_t far_grid = static_cast<uint32_t>(sm_count) * static_cast<uint32_t>(far_occ > 1 ? far_occ : 1);
    const uint32_t near_grid = static_cast<uint32_t>(sm_count) * static_cast<uint32_t>(near_occ > 1 ? near_occ : 1);
    const uint32_t finish_grid = static_cast<uint32_t>(sm_count) * 8u;
    const int crit_occ = trace_occupancy(kCriticalBlock, false, false);
    const uint32_t crit_grid = static_cast<uint32_t>(sm_count) * static_cast<uint32_t>(crit_occ > 1 ? crit_occ : 1);
    cudaError_t e = cudaSuccess;
    if (bands > 1) {
        if ((e = cudaEventRecord(static_cast<cudaEvent_t>(fork), s)) != cudaSuccess) return static_cast<int>(e);
        if ((e = cudaStreamWaitEvent(s2, static_cast<cudaEvent_t>(fork), 0)) != cudaSuccess) return static_cast<int>(e);
    }
    // bands of whole warps' worth of rays (multiples of 32); a band's hook is
    // enqueued after the next band's trace, so its work overlaps that trace
    const uint64_t per = ((n + bands - 1) / bands + 31) / 32 * 32;
    uint64_t begin = 0, prev_begin = 0, prev_count = 0;
    cudaStream_t prev_stream = nullptr;
    for (uint32_t b = 0; b < bands && begin < n && e == cudaSuccess; ++b) {
        const uint64_t count = (n - begin < per) ? n - begin : per;
        cudaStream_t sb = (b & 1u) ? s2 : s;
        const bool crit_beside = bands == 1 && buf.crit_stream && buf.crit_fork && buf.crit_join;
        e = enqueue_band(base, buf, begin, count, buf.counters + kBandCounterBytes * b, far_grid, far_block, near_grid,
                         finish_grid, crit_grid, crit_beside, sb);
        if (e == cudaSuccess && after_band && prev_stream)
            e = static_cast<cudaError_t>(after_band(hook_ctx, prev_begin, prev_count, prev_stream));
        prev_begin = begin;
        prev_count = count;
        prev_stream = sb;
        begin += count;
    }
    if (e == cudaSuccess && after_band && prev_stream)
        e = static_cast<cudaError_t>(after_band(hook_ctx, prev_begin, prev_count, prev_stream));
    if (e != cudaSuccess) return static_cast<int>(e);
    if (bands > 1) {
        if ((e = cudaEventRecord(static_cast<cudaEvent_t>(join), s2)) != cudaSuccess) return static_cast<int>(e);
        e = cudaStreamWaitEvent(s, static_cast<cudaEvent_t>(join), 0);
    }
    return static_cast<int>(e);
}

void launch_trace(const TraceArgs& args, uint32_t grid, uint32_t block, bool mixed, bool rolled, void* stream) {
    void* params[] = {const_cast<TraceArgs*>(&args)};
    // hydro model 2: the FP64 straight-line tracer in 128-thread blocks
    const int cont = args.cont.vol ? 2 : (args.cont.cross ? 1 : 0);
    block = (cont == 2) ? 128u : kernel_block(block, mixed, rolled);
    cudaLaunchKernel(kernel_for(block, mixed, rolled, cont), dim3(grid), dim3(block), params, 0,
                     static_cast<cudaStream_t>(stream));
}

rt_launch_config resolve_launch_config(rt_launch_config c, bool mixed) {
    if (c.block_size != 64 && c.block_size != 128 && c.block_size != 256) c.block_size = 128;
    c.fp64_rolled = c.fp64_rolled ? 1u : 0u;
    c.mixed_single_kernel = c.mixed_single_kernel ? 1u : 0u;
    c.block_size = kernel_block(c.block_size, mixed, c.fp64_rolled != 0);
    const int occ = trace_occupancy(c.block_size, mixed, c.fp64_rolled != 0);
    if (c.ctas_per_sm == 0 || static_cast<int>(c.ctas_per_sm) > occ) c.ctas_per_sm = occ > 1 ? occ : 1;
    // defaults from the autotuner on B200: whole-warp refills of 32 consecutive rays
    if (c.refill_threshold == 0 || c.refill_threshold > 32) c.refill_threshold = 32;
    if (c.rays_per_thread == 0 || c.rays_per_thread > 64) c.rays_per_thread = 1;
    return c;
}

}  // namespace relsim
