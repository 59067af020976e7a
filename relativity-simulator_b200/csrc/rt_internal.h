// rt_internal.h -- structures shared by the host code and the tracer kernels.
#pragma once

#include <cstdint>

#include "relsim_cuda.h"

namespace relsim {

// Bundle flags.
enum : uint32_t {
    BF_DISK = 1u << 0,          // thin disk present
    BF_EARLY_CAPTURE = 1u << 1, // Carter early capture allowed
    BF_MIXED = 1u << 2          // mixed-precision stages
};

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
    int32_t pad0;
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

// Device counters of one launch.
enum StatIndex { ST_RAYS = 0, ST_ATTEMPTS, ST_ACCEPTED, ST_RHS, ST_FP64_ATTEMPTS, ST_COUNT };

struct TraceArgs {
    const BundleDesc* bundles;
    uint32_t n_bundles;
    uint32_t refill_threshold;
    uint32_t claim;             // rays a warp claims per global atomic
    uint32_t pad;
    uint64_t total_rays;
    unsigned long long* queue;  // [0]: next unclaimed ray
    unsigned long long* stats;  // [ST_COUNT]
    OutPtrs out;
};

// Host-side helpers implemented in rt_bundle.cpp.
void build_bundle(const rt_camera& cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                  uint64_t ray_begin, uint64_t out_offset, BundleDesc& b);
double kerr_isco_radius(double m, double a);
// Row window of a camera (vulkan_compute_executor.hpp:1415-1426): first row and
// row count; count 0 in the camera means every row from the offset on.
void row_window(const rt_camera& c, uint32_t& row0, uint32_t& nrows);

// Tracer launch helpers implemented in rt_trace.cu.
void launch_trace(const TraceArgs& args, uint32_t grid, uint32_t block, bool mixed, bool rolled, void* stream);
int trace_occupancy(uint32_t block, bool mixed, bool rolled);
uint32_t kernel_block(uint32_t block, bool mixed, bool rolled);
// Launch shape with defaults filled in and limits applied for one precision.
rt_launch_config resolve_launch_config(rt_launch_config c, bool mixed);

}  // namespace relsim
