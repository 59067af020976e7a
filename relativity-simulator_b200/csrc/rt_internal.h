// rt_internal.h -- structures shared by the host code and the tracer kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include "relsim_cuda.h"
#include "rt_sky_profile.h"

namespace relsim {

// rt_ray_out as an array of pointers: its fields in declaration order and their
// element sizes
constexpr int kRayFields = 18;
constexpr size_t kRayFieldBytes[kRayFields] = {4, 4, 4, 4, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 4};
static_assert(sizeof(rt_ray_out) == kRayFields * sizeof(void*), "rt_ray_out is an array of pointers");

// Bundle flags.
enum : uint32_t {
    BF_DISK = 1u << 0,          // thin disk present
    BF_EARLY_CAPTURE = 1u << 1, // Carter early capture allowed
    BF_MIXED = 1u << 2          // mixed-precision stages
};

// Mixed mode: the near-critical band (M, distance of a ray's constants from
// the critical curve) of a camera that does not set one.  Rays inside it are
// traced in FP64 from their first step, at a tolerance graded with their
// distance from the curve.
constexpr float kDefaultCriticalBand = 1.0f;

// Per-camera constants, precomputed once on the host in FP64 (the same
// operations the reference performs per pixel that do not depend on the pixel:
// software_compute_engine.hpp:3790-3803 and :3902-3912, the observer's
// Kerr-Schild position and static-observer tetrad of
// kerr_schild_null_integrator.hpp:47-54, 142-177).
struct alignas(16) BundleDesc {
    // ray indexing
    uint64_t ray_begin;   // first global ray index of the bundle
    uint64_t out_offset;  // output element of the bundle's first ray
    uint32_t width, height;
    uint32_t col0, ncols;
    uint32_t row0, nrows;
    uint32_t max_steps;
    uint32_t flags;
    // camera
    double aspect, tan_half_fov;
    double fwd[3], rgt[3], up[3];
    double st, ct, sp, cp;  // sin/cos of the observer's theta and phi
    double x0[3];           // observer position, Kerr-Schild Cartesian
    double u0, two_h;       // static observer: u^t and 2H at x0
    double kf[3];           // Kerr-Schild null vector at x0
    double e[3][4];         // Gram-Schmidt spatial tetrad at x0
    double phi_start;       // unwrapped azimuth at the observer
    double raw_phi0;        // atan2(y, x) - atan2(a, r) at the observer
    int32_t wind0;          // phi_start = raw_phi0 + 2 pi wind0
    float critical_band;    // mixed mode: near-critical band in M (<= 0: none)
    // metric and integration
    double m, a, rh;
    double r_capture, r_esc, r_in, r_out, r_early;
    double rtol, atol, cap_c, h0, proj_tol;
    double fp64_radius;     // mixed mode: FP64 inside this radius
};

// Device output pointers (SoA record + optional 32-byte pixels).
struct OutPtrs {
    rt_pixel_out* pixels;
    rt_ray_out rays;
};

// Translucent-disk continuation outputs (structure of arrays, `stride`
// elements each, indexed like the record): the tracer records each disk
// crossing k < kMaxCrossings of a ray (r, phi, g at the crossing), and in
// info how many crossings it recorded, the class the ray ended with and
// whether its last point lay inside 3 r_s; the shading pass composes the
// pixel from them.  cross == nullptr: the tracer ends a ray at its first hit.
constexpr uint32_t kMaxCrossings = 8;
enum : uint32_t {
    CI_COUNT_MASK = 0xffu,  // bits 0..7: crossings recorded
    CI_FATE_SHIFT = 8u,     // bits 8..11: RT_RAY_* class at the ray's end
    CI_INSIDE_3RS = 1u << 12  // last point inside 3 r_s (6 M; multi-source: within 6 m of a source)
};
struct ShadeDesc;
struct ContOut {
    double* cross;    // [3 * kMaxCrossings][stride]: r_k at [3k], phi_k at [3k + 1], g_k at [3k + 2]
    uint32_t* info;   // [stride]
    uint64_t stride;
    uint32_t* body;   // multi-source: [stride], source of crossing k in bits 4k..4k+3 (else null)
    double* exit;     // Boyer-Lindquist and multi-source tracers, sky on: [3][stride], the
                      // sky-lookup direction at the ray's end (else null)
    double* tail;     // Kerr-Schild tracers, sky on: [stride][TL_COUNT], the ray's end (else null)
    double* vol;      // hydro model 2 (Kerr-Schild FP64 tracer): [stride][VL_COUNT], the light the
                      // ray gathered in the Fishbone-Moncrief torus (else null)
    const ShadeDesc* shade;  // with vol: the torus and the disk profile (device)
};
// The torus's light along a ray, gathered by the tracer step by step (every
// field 0 before the ray's first emitting segment): radiance r, g, b, the
// throughput left, the redshift of the last segment, and 1 once a segment
// emitted.
enum VolField : int { VL_R = 0, VL_G, VL_B, VL_THR, VL_Z, VL_HIT, VL_COUNT };
// The end of a Kerr-Schild ray's trace as its tracer leaves it for the shading
// pass, which derives the sky-lookup direction from it in parallel over the rays
// rather than on the tracer's divergent end path: the last step's end points and
// derivatives, its length, the threshold radius the end is interpolated to (0:
// the end is the point at TL_Y1) and the hole's mass and spin; one 224-byte
// record per ray, written by the ray's lane alone.
enum TailField : int { TL_Y0 = 0, TL_F0 = 6, TL_Y1 = 12, TL_F1 = 18, TL_H = 24, TL_TARGET, TL_M, TL_A, TL_COUNT };

// Device counters of one launch.
enum StatIndex { ST_RAYS = 0, ST_ATTEMPTS, ST_ACCEPTED, ST_RHS, ST_FP64_ATTEMPTS, ST_COUNT };

// Parked ray state of the two-pass mixed tracer: structure of arrays with one
// slot per ray of the launch, indexed by the ray's launch index.
enum ParkD : int { PD_Y = 0, PD_H = 6, PD_LAMBDA, PD_DH, PD_LZ0, PD_Q0, PD_COUNT };
enum ParkU : int { PU_ACC = 0, PU_REJ, PU_FLAGS, PU_GUARD, PU_WIND, PU_MISC, PU_LNP, PU_COUNT };
// PU_MISC bits
enum : uint32_t {
    PM_HAS_HIST = 1u,    // bit 0: PI30 history present
    PM_EARLY_SHIFT = 2u, // bits 2..3: Carter early-capture state + 1
    PM_CROSS_SHIFT = 5u  // bits 5..9: disk crossings so far (translucent-disk continuation)
};

struct ParkBuf {
    double* d;    // [PD_COUNT][n]
    uint32_t* u;  // [PU_COUNT][n]
    uint64_t n;   // slots
};

// Passes of the launch.  PASS_SINGLE: one kernel traces every ray to the end.
// The two-pass mixed tracer alternates an FP32 far-zone pass and an FP64
// near-zone pass; rays move between them through queues of launch indices.
enum TracePass : int { PASS_SINGLE = 0, PASS_FAR = 1, PASS_NEAR = 2 };

struct TraceArgs {
    const BundleDesc* bundles;
    uint32_t n_bundles;
    uint32_t refill_threshold;
    uint32_t claim;             // rays a warp claims per global atomic
    uint32_t pad;
    uint64_t total_rays;
    unsigned long long* queue;  // [0]: next unclaimed ray (or queue entry)
    unsigned long long* stats;  // [ST_COUNT]
    OutPtrs out;
    // two-pass mixed tracer (zero for PASS_SINGLE launches)
    uint64_t ray_base;          // far pass from pixels: launch index of this band's first ray
    uint32_t from_pixels;       // far pass: rays start at their pixels
    uint32_t allow_exit;        // near pass: rays leaving the near zone go back to the far pass
    const uint32_t* in_queue;   // launch indices of the rays to resume
    const uint32_t* in_count;
    uint32_t* out_queue;        // launch indices parked for the other pass
    uint32_t* out_count;
    uint32_t* finish_queue;     // disk hits parked with their root point for the finish pass
    uint32_t* finish_count;
    uint32_t* crit_queue;       // first far pass: near-critical rays, for the critical pass
    uint32_t* crit_count;
    ParkBuf park;
    // translucent-disk continuation (single-camera launches with shading): the
    // crossings' outputs; cross null: off
    ContOut cont;
};

// Multi-source Kerr-Schild superposition: per-source frame (source 0 is the
// camera's hole at the origin), as build_multi_source_data
// (software_compute_engine.hpp:2738-2798) builds it.
constexpr uint32_t kMaxSources = 16;
struct alignas(16) MsSource {
    double pos[3], m;
    double axis[3], a;
    double fx[3], rh;
    double fy[3], req;
    double disk_in, disk_out;  // disk_in < 0: no disk
    double pad0, pad1;
};

// Per-camera constants of a multi-source bundle.
struct alignas(16) MsDesc {
    uint64_t ray_begin, out_offset;
    uint32_t width, height, col0, ncols, row0, nrows;
    uint32_t max_steps, src_begin, src_count, pad0;
    double aspect, tan_half_fov;
    double fwd[3], rgt[3], up[3];
    double x0[3];     // observer, Cartesian point of (r, theta, phi)
    double phi0;      // atan2(y0, x0)
    double rtol, atol, cap_c, h0, proj_tol, r_esc, capture_scale;
};

struct MsArgs {
    const MsDesc* bundles;
    const MsSource* sources;
    uint32_t n_bundles;
    uint32_t refill_threshold;
    uint32_t claim;
    uint32_t pad;
    uint64_t total_rays;
    unsigned long long* queue;
    unsigned long long* stats;
    OutPtrs out;
    ContOut cont;  // translucent-disk continuation (shaded dispatches), else null
};

// Per-camera constants of the Boyer-Lindquist Kerr-Newman tracer, precomputed
// on the host in FP64: the pinhole camera, the observer's position and ZAMO
// tetrad (observer_tetrad.hpp:82-100; the tetrad is diagonal in (r, theta,
// phi) apart from e0's phi component), metric and integration constants.
struct alignas(16) BlDesc {
    uint64_t ray_begin, out_offset;
    uint32_t width, height, col0, ncols, row0, nrows;
    uint32_t max_steps, flags, pad0, pad1;
    double aspect, tan_half_fov;
    double fwd[3], rgt[3], up[3];
    double st, ct, sp, cp;          // sin/cos of the observer's theta and phi
    double r_obs, th_obs, ph_obs;
    double e0_t, e0_phi;            // ZAMO e0 = (1/alpha, 0, 0, omega/alpha)
    double e_r, e_th, e_ph;         // 1/sqrt(g_rr), 1/sqrt(g_thth), 1/sqrt(g_phiphi)
    double m, a, q2, rh;
    double r_capture, r_esc, r_in, r_out, r_early;
    double rtol, atol, cap_c, h0, proj_tol;
};

struct BlArgs {
    const BlDesc* bundles;
    uint32_t n_bundles;
    uint32_t refill_threshold;
    uint32_t claim;
    uint32_t pad;
    uint64_t total_rays;
    unsigned long long* queue;
    unsigned long long* stats;
    OutPtrs out;
    // translucent-disk continuation (shaded dispatches): the crossings' outputs;
    // cross null: off
    ContOut cont;
};

// Per-camera constants of the pixel shading pass (rt_shade.cu): the resolved
// disk profile, the disk's geometry, the Novikov-Thorne flux normalisation and
// its Page-Thorne roots, and the spectral table of the blackbody colour
// (33 trapezoid nodes over 380-780 nm, weights = node weight x CIE 1931 fit).
struct alignas(16) ShadeDesc {
    float profile[32];
    double mass, disk_spin, inner, outer, time, detail, exposure;
    double pattern_omega;                 // orbital angular velocity at sqrt(inner outer)
    double nt_flux_peak, nt_rate_factor;  // Novikov-Thorne: peak flux over the disk, rate^(1/4)
    double nt_m, nt_a_star, nt_x0, nt_x1, nt_x2, nt_x3, nt_r_isco;
    uint32_t hydro_model, tonemap, sky_on, pad1;
    double lambda_um[33];
    double weight[33][3];
    double fov;      // the camera's field of view (the sky's level of detail)
    SkyProfile sky;  // the procedural sky, read when sky_on
    // hydro model 2, the Fishbone-Moncrief torus: the hole (mass, clamped spin,
    // horizon), l and W_in, the peak enthalpy, the sampled radii, the density
    // exponent 1 / (gamma - 1), kappa (optical depth per M at peak enthalpy) and
    // samples per M of chord
    double fm_m, fm_a, fm_rh, fm_l, fm_w_in, fm_h_max, fm_inner, fm_outer, fm_exponent, fm_kappa, fm_density;
    uint32_t fm_valid, pad2;
};

// Build the shading constants of a camera; false if the settings are not
// supported (hydro model above 2, sky_enabled above 1).
bool build_shade_desc(const rt_camera& cam, const rt_shading& s, ShadeDesc& d);
void build_source_shade_desc(const ShadeDesc& base, const float* profile, double mass, double spin, double inner,
                             double outer, ShadeDesc& d);
// Shade n rays: pixels[i].rgba from the record's status, r_hit, phi and g.
void launch_shade(const ShadeDesc* desc, const uint32_t* status, const double* r_hit, const double* phi,
                  const double* g, ContOut cont, rt_pixel_out* pixels, uint64_t n, void* stream);

// Host-side helpers implemented in rt_bundle.cpp.
// Boyer-Lindquist bundle of a camera window (metric_form RT_METRIC_BOYER_LINDQUIST).
void build_bl_bundle(const rt_camera& cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                     uint64_t ray_begin, uint64_t out_offset, BlDesc& b);
// Outer horizon r_+ = M + sqrt(M^2 - a^2 - Q^2) (M when the root is imaginary).
double kn_horizon(double m, double a, double q);
// Source table of a multi-source camera: the camera's hole and up to 15
// sources; returns the count.
uint32_t build_ms_sources(const rt_camera& cam, const rt_source* src, uint32_t n, MsSource* out);
void build_ms_bundle(const rt_camera& cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                     uint64_t ray_begin, uint64_t out_offset, uint32_t src_begin, uint32_t src_count, MsDesc& b);
void build_bundle(const rt_camera& cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                  uint64_t ray_begin, uint64_t out_offset, BundleDesc& b);
double kerr_isco_radius(double m, double a);
// Row window of a camera (vulkan_compute_executor.hpp:1415-1426): first row and
// row count; count 0 in the camera means every row from the offset on.
void row_window(const rt_camera& c, uint32_t& row0, uint32_t& nrows);

// Tracer launch helpers implemented in rt_trace.cu.
void launch_trace(const TraceArgs& args, uint32_t grid, uint32_t block, bool mixed, bool rolled, void* stream);
// One pass of the two-pass mixed tracer (PASS_FAR or PASS_NEAR).
void launch_trace_pass(const TraceArgs& args, int pass, uint32_t grid, uint32_t block, void* stream);
int trace_pass_occupancy(int pass, uint32_t block);

// Device buffers of the two-pass mixed tracer for n rays.
struct TwoPassBuffers {
    ParkBuf park;       // parked state, n slots
    uint32_t* queues;   // 4n entries: per band near, far, finish and near-critical queues
    char* counters;     // kBandCounterBytes per band (up to kMaxBands): claim counters and queue counts
    // one band: the critical pass runs on this stream beside the near pass
    // (forked and joined with the two events); null: after it, on the band's
    void* crit_stream = nullptr;
    void* crit_fork = nullptr;
    void* crit_join = nullptr;
};
constexpr uint32_t kBandCounterBytes = 64;
constexpr uint32_t kMaxBands = 8;
// Bytes of park.d, park.u and queues for n rays.
uint64_t two_pass_state_bytes(uint64_t n);
// Work enqueued on a band's stream once the band is traced (rays [begin,
// begin + count) of the launch); returns a cudaError_t value.
typedef int (*BandHook)(void* ctx, uint64_t begin, uint64_t count, void* stream);

// Enqueue the rounds of the two-pass mixed tracer (memsets, launches and event
// records only, so it can be captured into a graph).  `base` carries the
// bundles, outputs, zeroed stats, the far pass's refill threshold and claim,
// and total_rays.  The rays are split into `bands` contiguous ranges traced
// alternately on `stream` and `stream2`, so that one band's near-pass tail
// overlaps the next band's far pass; fork and join (events created by the
// caller) bring stream2 into and out of the sequence.  bands = 1 uses
// `stream` alone.  Returns a cudaError_t value.
// after_band (optional) runs for each band after the next band's trace has been
// enqueued, so a band's copies can overlap the next band's trace.
int enqueue_two_pass(const TraceArgs& base, const TwoPassBuffers& buf, int sm_count, uint32_t far_block,
                     void* stream, void* stream2, void* fork, void* join, uint32_t bands,
                     BandHook after_band = nullptr, void* hook_ctx = nullptr);
int trace_occupancy(uint32_t block, bool mixed, bool rolled);
uint32_t kernel_block(uint32_t block, bool mixed, bool rolled);
// Launch shape with defaults filled in and limits applied for one precision.
rt_launch_config resolve_launch_config(rt_launch_config c, bool mixed);

// Multi-source tracer (rt_multi.cu).
void launch_ms_trace(const MsArgs& args, uint32_t grid, void* stream);
uint32_t ms_trace_grid(int sm_count);

// Boyer-Lindquist Kerr-Newman tracer (rt_bl.cu).
void launch_bl_trace(const BlArgs& args, uint32_t grid, void* stream);
uint32_t bl_trace_grid(int sm_count);

}  // namespace relsim
