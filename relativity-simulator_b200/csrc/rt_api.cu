// rt_api.cu -- C ABI of the tracer (include/relsim_cuda.h).
//
// Host side of the drop-in backend: VulkanComputeExecutor's lifetime,
// dispatch_and_readback and dispatch_tile_and_readback
// (vulkan_compute_executor.hpp:983-1464) over the persistent CUDA tracer.
// Device buffers are owned by the handle and grow on demand
// (ensure_output_capacity, vulkan_compute_executor.hpp:400); calls on one
// handle are serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "relsim_cuda.h"
#include "rt_internal.h"

namespace relsim {
double measure_fma_peak(bool fp64, int sm_count, cudaStream_t stream, float* ms_out);
}  // namespace relsim

using namespace relsim;

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct rt_handle {
    int device = -1;
    int sm_count = 0;
    bool ready = false;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;          // second stream of banded host dispatches
    cudaStream_t stream3 = nullptr;          // the mixed tracer's critical pass, beside its near passes
    cudaEvent_t ev_cfork = nullptr, ev_cjoin = nullptr;
    cudaStream_t copy_stream = nullptr;      // their device-to-host copies
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t band_ev[8] = {};             // band traced (and shaded): its copies may start
    std::string error;
    rt_launch_config cfg{};
    // device scratch
    DevBuf bundles, queue, stats;
    DevBuf park_d, park_u, pass_queues;  // two-pass mixed tracer: parked state, far/near queues
    DevBuf ms_desc, ms_sources;          // multi-source camera and source table
    DevBuf bl_desc;                      // Boyer-Lindquist camera
    DevBuf band_desc, band_queue;        // banded single-kernel host dispatches: per-band camera and counter
    DevBuf shade_desc;                   // pixel shading constants of the last shaded camera
    bool shade_on = false;               // rt_set_shading
    // translucent-disk continuation of a shaded dispatch: each ray's disk crossings
    // and how it ended, and what the launches pass the tracer
    DevBuf cont_cross, cont_info, cont_body, cont_exit, cont_tail, cont_vol;
    DevBuf ms_shade;  // multi-source shading: one descriptor per source
    ContOut cur_cont{};
    rt_shading shading{};
    DevBuf ray_fields[kRayFields];
    DevBuf pixels;
    // pinned staging of the bundle table
    BundleDesc* host_bundles = nullptr;
    size_t host_bundles_cap = 0;
    // last launch
    bool timed = false;
    // bundle graph cache
    cudaGraphExec_t graph = nullptr;
    uint32_t graph_n_bundles = 0;
    uint64_t graph_total = 0;
    OutPtrs graph_out{};
    rt_launch_config graph_cfg{};
};

namespace {

bool create_band_events(rt_handle* h) {
    for (cudaEvent_t& e : h->band_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
    return true;
}

rt_status fail(rt_handle* h, rt_status st, const std::string& msg) {
    if (h) h->error = msg;
    return st;
}

rt_status cuda_fail(rt_handle* h, cudaError_t e, const char* where) {
    cudaGetLastError();  // clear it: a later cudaGetLastError() must not report this call again
    if (h) {
        h->error = std::string(where) + ": " + cudaGetErrorString(e);
        if (e != cudaErrorMemoryAllocation && e != cudaErrorInvalidValue) h->ready = false;
    }
    return (e == cudaErrorMemoryAllocation) ? RT_ERR_OOM : RT_ERR_DEVICE;
}

#define RT_CUDA(h, call)                                          \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail((h), e_, #call); \
    } while (0)

rt_status ensure(rt_handle* h, DevBuf& b, size_t bytes) {
    if (b.bytes >= bytes) return RT_OK;
    if (b.ptr) {
        cudaFree(b.ptr);  // waits for the device: no launch still reads the old buffer
        // a captured bundle graph may hold the old address
        if (h->graph) cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    b.ptr = nullptr;
    b.bytes = 0;
    const size_t grow = std::max(bytes, b.bytes + b.bytes / 2);
    cudaError_t e = cudaMalloc(&b.ptr, grow);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(h, e, "cudaMalloc");
    }
    b.bytes = grow;
    return RT_OK;
}

void release(DevBuf& b) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

rt_status ensure_host_bundles(rt_handle* h, size_t n) {
    if (h->host_bundles_cap >= n) return RT_OK;
    if (h->host_bundles) {
        cudaFreeHost(h->host_bundles);
        if (h->graph) cudaGraphExecDestroy(h->graph);  // its upload node read the old staging buffer
        h->graph = nullptr;
    }
    h->host_bundles = nullptr;
    h->host_bundles_cap = 0;
    RT_CUDA(h, cudaMallocHost(&h->host_bundles, n * sizeof(BundleDesc)));
    h->host_bundles_cap = n;
    return RT_OK;
}

// Boyer-Lindquist form: a finite charge and a horizon, a^2 + Q^2 < M^2 after
// the spin clamp (the reference traces larger charges with r_+ = M, a radius
// that is no horizon).
bool bl_camera_valid(const rt_camera* c) {
    if (!std::isfinite(c->metric_charge)) return false;
    const double m = std::max(c->metric_mass, 1e-4);
    const double a = std::min(std::max(c->metric_spin, -0.999 * m), 0.999 * m);
    return m * m - a * a - c->metric_charge * c->metric_charge > 0.0;
}

bool is_bl(const rt_camera* c) { return c->metric_form == RT_METRIC_BOYER_LINDQUIST; }

bool camera_valid(const rt_camera* c) {
    return c && c->screen_width > 0 && c->screen_height > 0 && std::isfinite(c->metric_mass) &&
           (c->metric_form == RT_METRIC_KERR_SCHILD || (c->metric_form == RT_METRIC_BOYER_LINDQUIST && bl_camera_valid(c))) &&
           std::isfinite(c->metric_spin) && std::isfinite(c->field_of_view_rad) && c->field_of_view_rad > 0.0 &&
           c->field_of_view_rad < 3.14 && std::isfinite(c->escape_radius) && c->rtol > 0.0 && c->atol >= 0.0 &&
           c->step_cap_fraction > 0.0 && c->initial_step_fraction > 0.0 && c->capture_scale >= 1.0 &&
           c->max_integration_steps > 0 && std::isfinite(c->observer_position[1]) &&
           std::isfinite(c->observer_position[2]) && std::isfinite(c->observer_position[3]) &&
           !std::isnan(c->mixed_critical_band) &&
           (c->precision_mode == RT_PRECISION_FP64 || c->precision_mode == RT_PRECISION_MIXED);
}

rt_launch_config effective_cfg(const rt_handle* h, bool mixed) { return resolve_launch_config(h->cfg, mixed); }

// Parked-state and queue buffers of the two-pass tracer for `total` rays
// (allocated before any graph capture: allocation is not capturable).
rt_status ensure_two_pass(rt_handle* h, uint64_t total) {
    rt_status st;
    if ((st = ensure(h, h->park_d, sizeof(double) * PD_COUNT * total)) != RT_OK) return st;
    if ((st = ensure(h, h->park_u, sizeof(uint32_t) * PU_COUNT * total)) != RT_OK) return st;
    return ensure(h, h->pass_queues, sizeof(uint32_t) * 4 * total);
}

bool uses_two_pass(const rt_launch_config& c, bool mixed, uint64_t total) {
    return mixed && c.mixed_single_kernel == 0 && total <= 0xffffffffull;
}

rt_status launch_two_pass(rt_handle* h, uint32_t n_bundles, uint64_t total, const OutPtrs& out,
                          const rt_launch_config& c, cudaStream_t s, bool capturing, uint32_t bands = 1,
                          BandHook hook = nullptr, void* hook_ctx = nullptr) {
    if (!capturing) {
        const rt_status st = ensure_two_pass(h, total);
        if (st != RT_OK) return st;
    } else if (h->park_d.bytes < sizeof(double) * PD_COUNT * total ||
               h->park_u.bytes < sizeof(uint32_t) * PU_COUNT * total ||
               h->pass_queues.bytes < sizeof(uint32_t) * 4 * total) {
        return fail(h, RT_ERR_INVALID_ARG, "two-pass buffers not reserved before capture");
    }
    TraceArgs args{};
    args.bundles = static_cast<const BundleDesc*>(h->bundles.ptr);
    args.n_bundles = n_bundles;
    args.refill_threshold = c.refill_threshold;
    args.claim = 32u * c.rays_per_thread;
    args.total_rays = total;
    args.stats = static_cast<unsigned long long*>(h->stats.ptr);
    args.out = out;
    args.cont = h->cur_cont;
    TwoPassBuffers buf{};
    buf.park = ParkBuf{static_cast<double*>(h->park_d.ptr), static_cast<uint32_t*>(h->park_u.ptr), total};
    buf.queues = static_cast<uint32_t*>(h->pass_queues.ptr);
    buf.counters = static_cast<char*>(h->queue.ptr);
    buf.crit_stream = h->stream3;
    buf.crit_fork = h->ev_cfork;
    buf.crit_join = h->ev_cjoin;
    RT_CUDA(h, cudaMemsetAsync(h->stats.ptr, 0, sizeof(unsigned long long) * ST_COUNT, s));
    if (!capturing) RT_CUDA(h, cudaEventRecord(h->ev0, s));
    const bool banded = bands > 1 && !capturing;
    RT_CUDA(h, static_cast<cudaError_t>(enqueue_two_pass(
                   args, buf, h->sm_count, c.block_size, s, banded ? h->stream2 : nullptr,
                   banded ? h->ev_fork : nullptr, banded ? h->ev_join : nullptr, banded ? bands : 1, hook, hook_ctx)));
    if (!capturing) {
        RT_CUDA(h, cudaEventRecord(h->ev1, s));
        h->timed = true;
    }
    return RT_OK;
}

// Launch the tracer over `n` bundles already in h->bundles (device).  The
// timing events bracket the launch unless it is being captured into a graph
// (an event recorded on a capturing stream only orders the capture; the graph
// launch is bracketed instead).
rt_status launch(rt_handle* h, uint32_t n_bundles, uint64_t total, const OutPtrs& out, bool mixed, cudaStream_t s,
                 bool capturing = false) {
    const rt_launch_config c = effective_cfg(h, mixed);
    if (uses_two_pass(c, mixed, total)) return launch_two_pass(h, n_bundles, total, out, c, s, capturing);
    TraceArgs args{};
    args.bundles = static_cast<const BundleDesc*>(h->bundles.ptr);
    args.n_bundles = n_bundles;
    args.refill_threshold = c.refill_threshold;
    args.claim = 32u * c.rays_per_thread;
    args.total_rays = total;
    args.queue = static_cast<unsigned long long*>(h->queue.ptr);
    args.stats = static_cast<unsigned long long*>(h->stats.ptr);
    args.out = out;
    args.cont = h->cur_cont;
    RT_CUDA(h, cudaMemsetAsync(h->queue.ptr, 0, sizeof(unsigned long long), s));
    RT_CUDA(h, cudaMemsetAsync(h->stats.ptr, 0, sizeof(unsigned long long) * ST_COUNT, s));
    const uint32_t grid = static_cast<uint32_t>(h->sm_count) * c.ctas_per_sm;
    if (!capturing) RT_CUDA(h, cudaEventRecord(h->ev0, s));
    launch_trace(args, grid, c.block_size, mixed, c.fp64_rolled != 0, s);
    RT_CUDA(h, cudaGetLastError());
    if (!capturing) {
        RT_CUDA(h, cudaEventRecord(h->ev1, s));
        h->timed = true;
    }
    return RT_OK;
}

// Device SoA record in the handle's scratch for `n` rays: only the fields the
// caller asked for on the host.
rt_status scratch_rays(rt_handle* h, const rt_ray_out* host, size_t n, rt_ray_out& dev) {
    std::memset(&dev, 0, sizeof dev);
    if (!host) return RT_OK;
    void* const* hp = reinterpret_cast<void* const*>(host);
    void** dp = reinterpret_cast<void**>(&dev);
    for (int f = 0; f < kRayFields; ++f) {
        if (!hp[f]) continue;
        rt_status st = ensure(h, h->ray_fields[f], n * kRayFieldBytes[f]);
        if (st != RT_OK) return st;
        dp[f] = h->ray_fields[f].ptr;
    }
    return RT_OK;
}

rt_status copy_back(rt_handle* h, const rt_ray_out* host, const rt_ray_out& dev, rt_pixel_out* hpix,
                    const rt_pixel_out* dpix, size_t n, cudaStream_t s) {
    if (host) {
        void* const* hp = reinterpret_cast<void* const*>(host);
        void* const* dp = reinterpret_cast<void* const*>(&dev);
        for (int f = 0; f < kRayFields; ++f)
            if (hp[f]) RT_CUDA(h, cudaMemcpyAsync(hp[f], dp[f], n * kRayFieldBytes[f], cudaMemcpyDeviceToHost, s));
    }
    if (hpix) RT_CUDA(h, cudaMemcpyAsync(hpix, dpix, n * sizeof(rt_pixel_out), cudaMemcpyDeviceToHost, s));
    return RT_OK;
}

rt_status wait_stream(rt_handle* h, cudaStream_t s, double timeout_ms) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) return RT_OK;
        if (e != cudaErrorNotReady) return cuda_fail(h, e, "cudaStreamQuery");
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (timeout_ms > 0.0 && ms > timeout_ms) return fail(h, RT_ERR_TIMEOUT, "stream wait timed out");
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

rt_status bl_launch(rt_handle* h, const rt_camera* cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                    uint64_t out_offset, const OutPtrs& out, cudaStream_t s);
struct BandCopyCtx;
rt_status launch_banded_single(rt_handle* h, const rt_camera* cam, uint32_t col0, uint32_t ncols, uint32_t row0,
                               uint32_t nrows, uint64_t out_offset, const OutPtrs& out, BandCopyCtx& ctx);

// The record fields the shading pass reads (status, phi, r_hit, g), taken from
// the handle's scratch where the caller did not ask for them.
rt_status add_shade_fields(rt_handle* h, rt_ray_out& dev, size_t n) {
    void** dp = reinterpret_cast<void**>(&dev);
    const int fields[4] = {0, 6, 7, 8};
    const size_t elem[4] = {4, 8, 8, 8};
    for (int k = 0; k < 4; ++k) {
        const int f = fields[k];
        if (dp[f]) continue;
        const rt_status st = ensure(h, h->ray_fields[f], n * elem[k]);
        if (st != RT_OK) return st;
        dp[f] = h->ray_fields[f].ptr;
    }
    return RT_OK;
}

// Upload the shading constants of a camera (before the trace, on its stream).
rt_status shade_prepare(rt_handle* h, const rt_camera* cam, cudaStream_t s) {
    ShadeDesc d;
    if (!build_shade_desc(*cam, h->shading, d)) return fail(h, RT_ERR_INVALID_ARG, "unsupported shading settings");
    rt_status st;
    if ((st = ensure(h, h->shade_desc, sizeof(ShadeDesc))) != RT_OK) return st;
    // pageable descriptor: the copy is staged before the call returns
    RT_CUDA(h, cudaMemcpyAsync(h->shade_desc.ptr, &d, sizeof d, cudaMemcpyHostToDevice, s));
    return RT_OK;
}

// Turn on the translucent-disk continuation for the launches of a shaded
// dispatch of n rays: the tracers record each disk crossing and follow the ray
// on through the disk; the shading pass composes the crossings.
// The sky needs each ray's direction at its end: the Boyer-Lindquist and
// multi-source tracers write it (exit); the Kerr-Schild tracers leave the end of
// the trace to the shading pass (tail, `kerr_schild`).
rt_status begin_continuation(rt_handle* h, size_t n, bool bodies = false, bool kerr_schild = false,
                             cudaStream_t s = nullptr) {
    // hydro model 2: the single-hole tracers gather the torus's light into
    // per-ray records, zeroed here
    const bool volume = !bodies && h->shading.hydro_model == 2u;
    if (volume) {
        rt_status vs = ensure(h, h->cont_vol, sizeof(double) * VL_COUNT * n);
        if (vs != RT_OK) return vs;
        RT_CUDA(h, cudaMemsetAsync(h->cont_vol.ptr, 0, sizeof(double) * VL_COUNT * n, s));
    }
    double sky_enabled = 0.0;
    rt_sky_profile_get(&h->shading.sky, "enabled", &sky_enabled);
    const bool sky = h->shading.sky_enabled == 1u && sky_enabled != 0.0;
    const bool exit = sky && !kerr_schild, tail = sky && kerr_schild;
    rt_status st = ensure(h, h->cont_cross, sizeof(double) * 3 * kMaxCrossings * n);
    if (st == RT_OK) st = ensure(h, h->cont_info, sizeof(uint32_t) * n);
    if (st == RT_OK && bodies) st = ensure(h, h->cont_body, sizeof(uint32_t) * n);
    if (st == RT_OK && exit) st = ensure(h, h->cont_exit, sizeof(double) * 3 * n);
    if (st == RT_OK && tail) st = ensure(h, h->cont_tail, sizeof(double) * TL_COUNT * n);
    if (st != RT_OK) return st;
    h->cur_cont = ContOut{static_cast<double*>(h->cont_cross.ptr), static_cast<uint32_t*>(h->cont_info.ptr), n,
                          bodies ? static_cast<uint32_t*>(h->cont_body.ptr) : nullptr,
                          exit ? static_cast<double*>(h->cont_exit.ptr) : nullptr,
                          tail ? static_cast<double*>(h->cont_tail.ptr) : nullptr,
                          volume ? static_cast<double*>(h->cont_vol.ptr) : nullptr,
                          volume ? static_cast<const ShadeDesc*>(h->shade_desc.ptr) : nullptr};
    return RT_OK;
}

// Hydro model 2 traces the camera as the reference's image path does with the
// torus: no thin disk, the FP64 tracer at the camera's tolerances, and no
// early capture (a ray certain to be captured may still cross the torus on its
// way in).  Multi-source scenes keep the bodies' disks and lose the camera
// hole's, as the reference's multi-source path does (ms_dispatch_window).
bool volume_shading(const rt_handle* h, bool pixels) { return h->shade_on && pixels && h->shading.hydro_model == 2u; }
rt_camera volume_camera(const rt_camera& cam) {
    rt_camera c = cam;
    c.disk_outer_radius = 0.0;
    c.precision_mode = RT_PRECISION_FP64;
    c.early_capture = 0;
    return c;
}

void end_continuation_state(rt_handle* h) { h->cur_cont = ContOut{}; }

// Turns the continuation off when a dispatch returns, on every path.
struct ContinuationScope {
    rt_handle* h;
    ~ContinuationScope() { end_continuation_state(h); }
};

// Enqueue the shading pass over n traced rays (after the trace, same stream).
rt_status shade_launch(rt_handle* h, const rt_camera* cam, const rt_ray_out& dev, rt_pixel_out* pixels, size_t n,
                       cudaStream_t s, bool prepared = false) {
    rt_status st;
    if (!prepared && (st = shade_prepare(h, cam, s)) != RT_OK) return st;
    launch_shade(static_cast<const ShadeDesc*>(h->shade_desc.ptr), dev.status, dev.r_hit, dev.phi, dev.g, h->cur_cont,
                 pixels, n, s);
    RT_CUDA(h, cudaGetLastError());
    return RT_OK;
}

// Per-band work of a banded host dispatch: shade the band's rays on the band's
// stream, then copy its slice of the pixels and of every record field the
// caller asked for on the copy stream (once the band is done), so that no
// trace waits behind a copy.
struct BandCopyCtx {
    rt_handle* h;
    const rt_ray_out* host;
    rt_ray_out dev;
    rt_pixel_out* hpix;
    rt_pixel_out* dpix;
    uint64_t offset;  // output element of the launch's first ray
    bool shade;
    uint32_t band;    // next band event
    ContOut cont;     // translucent-disk continuation outputs (rgb null: none)
};

int band_copy_hook(void* vctx, uint64_t begin, uint64_t count, void* stream) {
    BandCopyCtx& c = *static_cast<BandCopyCtx*>(vctx);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t o = c.offset + begin;
    if (c.shade && c.dpix) {
        launch_shade(static_cast<const ShadeDesc*>(c.h->shade_desc.ptr), c.dev.status + o, c.dev.r_hit + o,
                     c.dev.phi + o, c.dev.g + o,
                     c.cont.cross ? ContOut{c.cont.cross + o, c.cont.info + o, c.cont.stride,
                                            c.cont.body ? c.cont.body + o : nullptr,
                                            c.cont.exit ? c.cont.exit + o : nullptr,
                                            c.cont.tail ? c.cont.tail + o * TL_COUNT : nullptr,
                                            c.cont.vol ? c.cont.vol + o * VL_COUNT : nullptr, c.cont.shade}
                                  : ContOut{},
                     c.dpix + o, count, s);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return static_cast<int>(e);
    }
    cudaEvent_t ev = c.h->band_ev[c.band++ % 8];
    cudaError_t e0 = cudaEventRecord(ev, s);
    if (e0 == cudaSuccess) e0 = cudaStreamWaitEvent(c.h->copy_stream, ev, 0);
    if (e0 != cudaSuccess) return static_cast<int>(e0);
    s = c.h->copy_stream;
    if (c.host) {
        void* const* hp = reinterpret_cast<void* const*>(c.host);
        void* const* dp = reinterpret_cast<void* const*>(&c.dev);
        for (int f = 0; f < kRayFields; ++f) {
            if (!hp[f]) continue;
            const size_t b = kRayFieldBytes[f];
            const cudaError_t e = cudaMemcpyAsync(static_cast<char*>(hp[f]) + o * b,
                                                  static_cast<const char*>(dp[f]) + o * b, count * b,
                                                  cudaMemcpyDeviceToHost, s);
            if (e != cudaSuccess) return static_cast<int>(e);
        }
    }
    if (c.hpix) {
        const cudaError_t e = cudaMemcpyAsync(c.hpix + o, c.dpix + o, count * sizeof(rt_pixel_out),
                                              cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) return static_cast<int>(e);
    }
    return static_cast<int>(cudaSuccess);
}

// Bands of a host dispatch on the two-pass tracer: each band's copies overlap
// the next band's trace (1 M rays and up).  Four: with every ray followed
// through the disk and the sky shaded, each band's pass tails cost more than
// the longer exposed copy of the last band (measured at 2048^2: 2 / 4 / 8 / 16
// bands 75.7 / 75.2 / 80.9 / 81.3 ms an image).
constexpr uint32_t kCopyBands = 4;
constexpr uint64_t kBandedMinRays = uint64_t{1} << 20;

// One host-buffer dispatch over a window (dispatch_and_readback semantics).
rt_status dispatch_window(rt_handle* h, const rt_camera* cam, uint32_t col0, uint32_t ncols, uint32_t row0,
                          uint32_t nrows, rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity,
                          const volatile int* cancel) {
    const size_t n = static_cast<size_t>(ncols) * nrows;
    if (n == 0) return fail(h, RT_ERR_INVALID_ARG, "empty window");
    if (capacity < n) return fail(h, RT_ERR_INVALID_ARG, "capacity smaller than the window");
    rt_status st = ensure_host_bundles(h, 1);
    if (st != RT_OK) return st;
    if ((st = ensure(h, h->bundles, sizeof(BundleDesc))) != RT_OK) return st;
    rt_ray_out dev{};
    if ((st = scratch_rays(h, rays, n, dev)) != RT_OK) return st;
    rt_pixel_out* dpix = nullptr;
    if (pixels) {
        if ((st = ensure(h, h->pixels, n * sizeof(rt_pixel_out))) != RT_OK) return st;
        dpix = static_cast<rt_pixel_out*>(h->pixels.ptr);
    }
    const bool shade = h->shade_on && pixels;
    ContinuationScope cont_scope{h};
    if (shade && (st = add_shade_fields(h, dev, n)) != RT_OK) return st;
    if (shade && (st = shade_prepare(h, cam, h->stream)) != RT_OK) return st;
    if (shade && (st = begin_continuation(h, n, false, !is_bl(cam), h->stream)) != RT_OK) return st;
    // bands of at most 2^24 rays; the cancel flag is polled between bands.  Each
    // band's shading and copies follow its trace; on the two-pass tracer a band
    // is traced in sub-bands whose copies overlap the next sub-band's trace.
    const uint64_t band_rows = std::max<uint64_t>(1, (uint64_t{1} << 24) / ncols);
    for (uint32_t r = 0; r < nrows; r += static_cast<uint32_t>(band_rows)) {
        if (cancel && *cancel) return fail(h, RT_ERR_CANCELLED, "cancelled");
        const uint32_t rows = static_cast<uint32_t>(std::min<uint64_t>(band_rows, nrows - r));
        const uint64_t offset = static_cast<uint64_t>(r) * ncols;
        const uint64_t launch_rays = static_cast<uint64_t>(rows) * ncols;
        BandCopyCtx ctx{h, rays, dev, pixels, dpix, offset, shade, 0, h->cur_cont};
        const bool two_pass = !is_bl(cam) && uses_two_pass(effective_cfg(h, cam->precision_mode == RT_PRECISION_MIXED),
                                                          cam->precision_mode == RT_PRECISION_MIXED, launch_rays);
        if (!two_pass && launch_rays >= kBandedMinRays && rows >= kCopyBands) {
            if ((st = launch_banded_single(h, cam, col0, ncols, row0 + r, rows, offset, OutPtrs{dpix, dev}, ctx)) !=
                RT_OK)
                return st;
            if ((st = wait_stream(h, h->stream, 0.0)) != RT_OK) return st;
            if ((st = wait_stream(h, h->copy_stream, 0.0)) != RT_OK) return st;
            continue;
        }
        if (is_bl(cam)) {
            if ((st = bl_launch(h, cam, col0, ncols, row0 + r, rows, offset, OutPtrs{dpix, dev}, h->stream)) != RT_OK)
                return st;
        } else {
            build_bundle(*cam, col0, ncols, row0 + r, rows, 0, offset, h->host_bundles[0]);
            RT_CUDA(h, cudaMemcpyAsync(h->bundles.ptr, h->host_bundles, sizeof(BundleDesc), cudaMemcpyHostToDevice,
                                       h->stream));
            const bool mixed = cam->precision_mode == RT_PRECISION_MIXED;
            const rt_launch_config c = effective_cfg(h, mixed);
            if (uses_two_pass(c, mixed, launch_rays) && launch_rays >= kBandedMinRays) {
                if ((st = launch_two_pass(h, 1, launch_rays, OutPtrs{dpix, dev}, c, h->stream, false, kCopyBands,
                                          band_copy_hook, &ctx)) != RT_OK)
                    return st;
                if ((st = wait_stream(h, h->stream, 0.0)) != RT_OK) return st;
                if ((st = wait_stream(h, h->copy_stream, 0.0)) != RT_OK) return st;
                continue;
            }
            if ((st = launch(h, 1, launch_rays, OutPtrs{dpix, dev}, mixed, h->stream)) != RT_OK) return st;
        }
        RT_CUDA(h, static_cast<cudaError_t>(band_copy_hook(&ctx, 0, launch_rays, h->stream)));
        if ((st = wait_stream(h, h->stream, 0.0)) != RT_OK) return st;
        if ((st = wait_stream(h, h->copy_stream, 0.0)) != RT_OK) return st;
    }
    return RT_OK;
}

// Enqueue a multi-source trace of the camera's row window (outputs: device).
rt_status ms_launch(rt_handle* h, const rt_camera* cam, const rt_source* src, uint32_t n_src, uint32_t row0,
                    uint32_t nrows, const OutPtrs& out, cudaStream_t s) {
    MsSource table[kMaxSources];
    const uint32_t count = build_ms_sources(*cam, src, n_src, table);
    MsDesc d;
    build_ms_bundle(*cam, 0, cam->screen_width, row0, nrows, 0, 0, 0, count, d);
    rt_status st;
    if ((st = ensure(h, h->ms_desc, sizeof(MsDesc))) != RT_OK) return st;
    if ((st = ensure(h, h->ms_sources, sizeof(table))) != RT_OK) return st;
    // pageable sources: each copy is staged before the call returns
    RT_CUDA(h, cudaMemcpyAsync(h->ms_desc.ptr, &d, sizeof d, cudaMemcpyHostToDevice, s));
    RT_CUDA(h, cudaMemcpyAsync(h->ms_sources.ptr, table, sizeof(MsSource) * count, cudaMemcpyHostToDevice, s));
    RT_CUDA(h, cudaMemsetAsync(h->queue.ptr, 0, sizeof(unsigned long long), s));
    RT_CUDA(h, cudaMemsetAsync(h->stats.ptr, 0, sizeof(unsigned long long) * ST_COUNT, s));
    const rt_launch_config c = effective_cfg(h, false);
    MsArgs args{};
    args.bundles = static_cast<const MsDesc*>(h->ms_desc.ptr);
    args.sources = static_cast<const MsSource*>(h->ms_sources.ptr);
    args.n_bundles = 1;
    args.refill_threshold = c.refill_threshold;
    args.claim = 32u * c.rays_per_thread;
    args.total_rays = static_cast<uint64_t>(cam->screen_width) * nrows;
    args.queue = static_cast<unsigned long long*>(h->queue.ptr);
    args.stats = static_cast<unsigned long long*>(h->stats.ptr);
    args.out = out;
    args.cont = h->cur_cont;
    RT_CUDA(h, cudaEventRecord(h->ev0, s));
    launch_ms_trace(args, ms_trace_grid(h->sm_count), s);
    RT_CUDA(h, cudaGetLastError());
    RT_CUDA(h, cudaEventRecord(h->ev1, s));
    h->timed = true;
    return RT_OK;
}

rt_status ms_check(rt_handle* h, const rt_camera* cam, const rt_source* src, uint32_t n_src) {
    if (!h->ready) return fail(h, RT_ERR_NOT_READY, "handle not ready");
    if (!camera_valid(cam)) return fail(h, RT_ERR_INVALID_ARG, "invalid camera");
    if (n_src > RT_MAX_SOURCES - 1) return fail(h, RT_ERR_INVALID_ARG, "at most 15 sources beside the camera's hole");
    if (n_src > 0 && !src) return fail(h, RT_ERR_INVALID_ARG, "null source table");
    for (uint32_t i = 0; i < n_src; ++i)
        if (!std::isfinite(src[i].mass) || !(src[i].mass > 0.0) || !std::isfinite(src[i].position[0]) ||
            !std::isfinite(src[i].position[1]) || !std::isfinite(src[i].position[2]))
            return fail(h, RT_ERR_INVALID_ARG, "invalid source");
    return RT_OK;
}

// Enqueue a Boyer-Lindquist trace of a camera window, its first ray written at
// element out_offset of the (device) outputs.
rt_status bl_launch(rt_handle* h, const rt_camera* cam, uint32_t col0, uint32_t ncols, uint32_t row0, uint32_t nrows,
                    uint64_t out_offset, const OutPtrs& out, cudaStream_t s) {
    BlDesc d;
    build_bl_bundle(*cam, col0, ncols, row0, nrows, 0, out_offset, d);
    rt_status st;
    if ((st = ensure(h, h->bl_desc, sizeof(BlDesc))) != RT_OK) return st;
    // pageable descriptor: the copy is staged before the call returns
    RT_CUDA(h, cudaMemcpyAsync(h->bl_desc.ptr, &d, sizeof d, cudaMemcpyHostToDevice, s));
    RT_CUDA(h, cudaMemsetAsync(h->queue.ptr, 0, sizeof(unsigned long long), s));
    RT_CUDA(h, cudaMemsetAsync(h->stats.ptr, 0, sizeof(unsigned long long) * ST_COUNT, s));
    const rt_launch_config c = effective_cfg(h, false);
    BlArgs args{};
    args.bundles = static_cast<const BlDesc*>(h->bl_desc.ptr);
    args.n_bundles = 1;
    args.refill_threshold = c.refill_threshold;
    args.claim = 32u * c.rays_per_thread;
    args.total_rays = static_cast<uint64_t>(ncols) * nrows;
    args.queue = static_cast<unsigned long long*>(h->queue.ptr);
    args.stats = static_cast<unsigned long long*>(h->stats.ptr);
    args.out = out;
    args.cont = h->cur_cont;
    RT_CUDA(h, cudaEventRecord(h->ev0, s));
    launch_bl_trace(args, bl_trace_grid(h->sm_count), s);
    RT_CUDA(h, cudaGetLastError());
    RT_CUDA(h, cudaEventRecord(h->ev1, s));
    h->timed = true;
    return RT_OK;
}

// A single-kernel host dispatch (the plain FP64 or single mixed Kerr-Schild
// tracer, or the Boyer-Lindquist tracer) in kCopyBands row bands: each band is
// one persistent launch with its own camera descriptor and work counter, the
// bands alternate between the handle's two streams, and each band's shading and
// copies (band_copy_hook) are enqueued after the next band's launch.
rt_status launch_banded_single(rt_handle* h, const rt_camera* cam, uint32_t col0, uint32_t ncols, uint32_t row0,
                               uint32_t nrows, uint64_t out_offset, const OutPtrs& out, BandCopyCtx& ctx) {
    const bool bl = is_bl(cam);
    const bool mixed = !bl && cam->precision_mode == RT_PRECISION_MIXED;
    const size_t desc_bytes = bl ? sizeof(BlDesc) : sizeof(BundleDesc);
    rt_status st;
    if ((st = ensure(h, h->band_desc, desc_bytes * kCopyBands)) != RT_OK) return st;
    if ((st = ensure(h, h->band_queue, sizeof(unsigned long long) * kCopyBands)) != RT_OK) return st;
    const rt_launch_config c = effective_cfg(h, mixed);
    cudaStream_t s = h->stream, s2 = h->stream2;
    RT_CUDA(h, cudaMemsetAsync(h->stats.ptr, 0, sizeof(unsigned long long) * ST_COUNT, s));
    RT_CUDA(h, cudaMemsetAsync(h->band_queue.ptr, 0, sizeof(unsigned long long) * kCopyBands, s));
    RT_CUDA(h, cudaEventRecord(h->ev0, s));
    RT_CUDA(h, cudaEventRecord(h->ev_fork, s));
    RT_CUDA(h, cudaStreamWaitEvent(s2, h->ev_fork, 0));
    const uint32_t per = (nrows + kCopyBands - 1) / kCopyBands;
    uint64_t prev_begin = 0, prev_count = 0;
    cudaStream_t prev_stream = nullptr;
    uint32_t b = 0;
    for (uint32_t r = 0; r < nrows; r += per, ++b) {
        const uint32_t rows = std::min(per, nrows - r);
        const uint64_t begin = static_cast<uint64_t>(r) * ncols;
        const uint64_t count = static_cast<uint64_t>(rows) * ncols;
        cudaStream_t sb = (b & 1u) ? s2 : s;
        char* dd = static_cast<char*>(h->band_desc.ptr) + desc_bytes * b;
        unsigned long long* q = static_cast<unsigned long long*>(h->band_queue.ptr) + b;
        // pageable descriptors: each copy is staged before the call returns
        if (bl) {
            BlDesc d;
            build_bl_bundle(*cam, col0, ncols, row0 + r, rows, 0, out_offset + begin, d);
            RT_CUDA(h, cudaMemcpyAsync(dd, &d, sizeof d, cudaMemcpyHostToDevice, sb));
            BlArgs args{};
            args.bundles = reinterpret_cast<const BlDesc*>(dd);
            args.n_bundles = 1;
            args.refill_threshold = c.refill_threshold;
            args.claim = 32u * c.rays_per_thread;
            args.total_rays = count;
            args.queue = q;
            args.stats = static_cast<unsigned long long*>(h->stats.ptr);
            args.out = out;
            args.cont = h->cur_cont;
            launch_bl_trace(args, bl_trace_grid(h->sm_count), sb);
        } else {
            BundleDesc d;
            build_bundle(*cam, col0, ncols, row0 + r, rows, 0, out_offset + begin, d);
            RT_CUDA(h, cudaMemcpyAsync(dd, &d, sizeof d, cudaMemcpyHostToDevice, sb));
            TraceArgs args{};
            args.bundles = reinterpret_cast<const BundleDesc*>(dd);
            args.n_bundles = 1;
            args.refill_threshold = c.refill_threshold;
            args.claim = 32u * c.rays_per_thread;
            args.total_rays = count;
            args.queue = q;
            args.stats = static_cast<unsigned long long*>(h->stats.ptr);
            args.out = out;
            args.cont = h->cur_cont;
            launch_trace(args, static_cast<uint32_t>(h->sm_count) * c.ctas_per_sm, c.block_size, mixed,
                         c.fp64_rolled != 0, sb);
        }
        RT_CUDA(h, cudaGetLastError());
        if (prev_stream) RT_CUDA(h, static_cast<cudaError_t>(band_copy_hook(&ctx, prev_begin, prev_count, prev_stream)));
        prev_begin = begin;
        prev_count = count;
        prev_stream = sb;
    }
    if (prev_stream) RT_CUDA(h, static_cast<cudaError_t>(band_copy_hook(&ctx, prev_begin, prev_count, prev_stream)));
    RT_CUDA(h, cudaEventRecord(h->ev_join, s2));
    RT_CUDA(h, cudaStreamWaitEvent(s, h->ev_join, 0));
    RT_CUDA(h, cudaEventRecord(h->ev1, s));
    h->timed = true;
    return RT_OK;
}

}  // namespace

extern "C" {

int rt_abi_version(void) { return RT_ABI_VERSION; }

// Shading descriptors of a multi-source scene: the camera's hole with
// rt_shading's resolved disk, each body with its own disk profile; every
// source shaded by the thin procedural model at detail 1 (trace_multi_source,
// software_compute_engine.hpp:3172-3185).
rt_status ms_shade_prepare(rt_handle* h, const rt_camera* cam, const rt_source* sources, uint32_t n_sources,
                           cudaStream_t s) {
    MsSource table[kMaxSources];
    const uint32_t count = build_ms_sources(*cam, sources, n_sources, table);
    ShadeDesc d[kMaxSources];
    ShadeDesc base;
    if (!build_shade_desc(*cam, h->shading, base)) return fail(h, RT_ERR_INVALID_ARG, "unsupported shading settings");
    build_source_shade_desc(base, nullptr, table[0].m, table[0].a, table[0].disk_in, table[0].disk_out, d[0]);
    for (uint32_t i = 1; i < count; ++i)
        build_source_shade_desc(base, reinterpret_cast<const float*>(&sources[i - 1].disk), table[i].m, table[i].a,
                                table[i].disk_in, table[i].disk_out, d[i]);
    rt_status st;
    if ((st = ensure(h, h->ms_shade, sizeof(ShadeDesc) * kMaxSources)) != RT_OK) return st;
    // pageable descriptors: the copy is staged before the call returns
    RT_CUDA(h, cudaMemcpyAsync(h->ms_shade.ptr, d, sizeof(ShadeDesc) * count, cudaMemcpyHostToDevice, s));
    return RT_OK;
}

// Trace a multi-source window into device outputs; shaded (handle shading on,
// pixels requested): every ray followed through the translucent disks and its
// crossings composed by the shading pass.
rt_status ms_dispatch_window(rt_handle* h, const rt_camera* cam, const rt_source* sources, uint32_t n_sources,
                             uint32_t row0, uint32_t nrows, const OutPtrs& out, cudaStream_t s) {
    const size_t n = static_cast<size_t>(cam->screen_width) * nrows;
    const bool shade = h->shade_on && out.pixels;
    rt_status st;
    ContinuationScope cont_scope{h};
    // hydro model 2: the reference's multi-source path draws no torus and turns
    // the camera hole's disk off (software_compute_engine.hpp:2752); the bodies'
    // disks stay
    rt_camera vc;
    if (volume_shading(h, out.pixels != nullptr)) {
        vc = *cam;
        vc.disk_outer_radius = 0.0;
        cam = &vc;
    }
    if (shade && (st = ms_shade_prepare(h, cam, sources, n_sources, s)) != RT_OK) return st;
    if (shade && (st = begin_continuation(h, n, true)) != RT_OK) return st;
    if ((st = ms_launch(h, cam, sources, n_sources, row0, nrows, out, s)) != RT_OK) return st;
    if (shade) {
        launch_shade(static_cast<const ShadeDesc*>(h->ms_shade.ptr), nullptr, nullptr, nullptr, nullptr, h->cur_cont,
                     out.pixels, n, s);
        RT_CUDA(h, cudaGetLastError());
    }
    return RT_OK;
}

rt_status rt_dispatch_multi(rt_handle* h, const rt_camera* cam, const rt_source* sources, uint32_t n_sources,
                            rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity) {
    if (!h) return RT_ERR_INVALID_ARG;
    rt_status st = ms_check(h, cam, sources, n_sources);
    if (st != RT_OK) return st;
    uint32_t row0, nrows;
    row_window(*cam, row0, nrows);
    const size_t n = static_cast<size_t>(cam->screen_width) * nrows;
    if (n == 0) return fail(h, RT_ERR_INVALID_ARG, "empty row window");
    if (capacity < n) return fail(h, RT_ERR_INVALID_ARG, "capacity smaller than the window");
    RT_CUDA(h, cudaSetDevice(h->device));
    rt_ray_out dev{};
    if ((st = scratch_rays(h, rays, n, dev)) != RT_OK) return st;
    rt_pixel_out* dpix = nullptr;
    if (pixels) {
        if ((st = ensure(h, h->pixels, n * sizeof(rt_pixel_out))) != RT_OK) return st;
        dpix = static_cast<rt_pixel_out*>(h->pixels.ptr);
    }
    if ((st = ms_dispatch_window(h, cam, sources, n_sources, row0, nrows, OutPtrs{dpix, dev}, h->stream)) != RT_OK)
        return st;
    if ((st = copy_back(h, rays, dev, pixels, dpix, n, h->stream)) != RT_OK) return st;
    return wait_stream(h, h->stream, 0.0);
}

rt_status rt_dispatch_multi_device(rt_handle* h, const rt_camera* cam, const rt_source* sources, uint32_t n_sources,
                                   rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity, void* stream) {
    if (!h) return RT_ERR_INVALID_ARG;
    rt_status st = ms_check(h, cam, sources, n_sources);
    if (st != RT_OK) return st;
    if (pixels && (reinterpret_cast<uintptr_t>(pixels) & 15u)) return fail(h, RT_ERR_INVALID_ARG, "pixels not 16-byte aligned");
    uint32_t row0, nrows;
    row_window(*cam, row0, nrows);
    const size_t n = static_cast<size_t>(cam->screen_width) * nrows;
    if (n == 0) return fail(h, RT_ERR_INVALID_ARG, "empty row window");
    if (capacity < n) return fail(h, RT_ERR_INVALID_ARG, "capacity smaller than the window");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    RT_CUDA(h, cudaSetDevice(h->device));
    return ms_dispatch_window(h, cam, sources, n_sources, row0, nrows, OutPtrs{pixels, rays ? *rays : rt_ray_out{}},
                              s);
}

double rt_kerr_isco_radius(double mass, double spin) { return kerr_isco_radius(mass, spin); }

int rt_is_platform_supported(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    for (int d = 0; d < n; ++d) {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10 && p.minor == 0) return 1;
    }
    return 0;
}

rt_status rt_create(rt_handle** out, int device_ordinal) {
    if (!out) return RT_ERR_INVALID_ARG;
    *out = nullptr;
    rt_handle* h = new (std::nothrow) rt_handle();
    if (!h) return RT_ERR_OOM;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || device_ordinal < 0 || device_ordinal >= n) {
        cudaGetLastError();
        delete h;
        return RT_ERR_DEVICE;
    }
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, device_ordinal) != cudaSuccess || p.major != 10 || p.minor != 0) {
        delete h;
        return RT_ERR_DEVICE;  // built for sm_100a only
    }
    h->device = device_ordinal;
    h->sm_count = p.multiProcessorCount;
    if (cudaSetDevice(device_ordinal) != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream3, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_cfork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_cjoin, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess || !create_band_events(h)) {
        cudaGetLastError();
        rt_destroy(h);
        return RT_ERR_DEVICE;
    }
    if (ensure(h, h->queue, kBandCounterBytes * kMaxBands) != RT_OK || ensure(h, h->stats, 256) != RT_OK) {
        rt_destroy(h);
        return RT_ERR_OOM;
    }
    h->ready = true;
    *out = h;
    return RT_OK;
}

void rt_destroy(rt_handle* h) {
    if (!h) return;
    if (h->device >= 0) cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    release(h->bundles);
    release(h->ms_desc);
    release(h->ms_sources);
    release(h->bl_desc);
    release(h->band_desc);
    release(h->band_queue);
    release(h->shade_desc);
    release(h->ms_shade);
    release(h->cont_cross);
    release(h->cont_info);
    release(h->cont_body);
    release(h->cont_exit);
    release(h->cont_tail);
    release(h->cont_vol);
    release(h->park_d);
    release(h->park_u);
    release(h->pass_queues);
    release(h->queue);
    release(h->stats);
    release(h->pixels);
    for (auto& b : h->ray_fields) release(b);
    if (h->host_bundles) cudaFreeHost(h->host_bundles);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_cfork) cudaEventDestroy(h->ev_cfork);
    if (h->ev_cjoin) cudaEventDestroy(h->ev_cjoin);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    for (cudaEvent_t& e : h->band_ev)
        if (e) cudaEventDestroy(e);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    if (h->stream2) cudaStreamDestroy(h->stream2);
    if (h->stream3) cudaStreamDestroy(h->stream3);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int rt_is_ready(const rt_handle* h) { return (h && h->ready) ? 1 : 0; }

const char* rt_last_error(const rt_handle* h) { return h ? h->error.c_str() : "null handle"; }

void rt_camera_defaults(rt_camera* c) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->field_of_view_rad = 12.0 * 3.14159265358979323846 / 180.0;
    c->metric_mass = 1.0;
    c->metric_spin = 0.94;
    c->escape_radius = 1000.0;
    c->capture_scale = 1.01;
    c->disk_inner_radius = 0.0;
    c->disk_outer_radius = 20.0;
    c->rtol = 1e-10;
    c->atol = 1e-10;
    c->step_cap_fraction = 0.1;
    c->initial_step_fraction = 0.01;
    c->projection_tol = 1e-12;
    c->mixed_fp64_radius = 0.0;
    c->mixed_critical_band = 0.0;
    c->screen_width = 2048;
    c->screen_height = 2048;
    c->max_integration_steps = 20000;
    c->early_capture = 1;
    c->precision_mode = RT_PRECISION_FP64;
    rt_camera_look_at_hole(c, 100.0, 17.0 * 3.14159265358979323846 / 180.0, 0.0);
}

void rt_camera_look_at_hole(rt_camera* c, double r, double theta, double phi) {
    if (!c) return;
    const double st = std::sin(theta), ct = std::cos(theta), sp = std::sin(phi), cp = std::cos(phi);
    const double er[3] = {st * cp, st * sp, ct};
    const double eth[3] = {ct * cp, ct * sp, -st};
    const double eph[3] = {-sp, cp, 0.0};
    c->observer_position[0] = 0.0;
    c->observer_position[1] = r;
    c->observer_position[2] = theta;
    c->observer_position[3] = phi;
    c->tetrad_e1[0] = c->tetrad_e2[0] = c->tetrad_e3[0] = 0.0;
    for (int i = 0; i < 3; ++i) {
        c->tetrad_e1[1 + i] = -er[i];
        c->tetrad_e2[1 + i] = eph[i];
        c->tetrad_e3[1 + i] = -eth[i];
    }
}

void rt_shading_defaults(rt_shading* s) {
    if (!s) return;
    std::memset(s, 0, sizeof *s);
    // GpuDiskProfile's defaults (gpu_types.hpp:42-75), in its field order
    const float disk[32] = {1.0f, 1.0f, 24.0f, 9500.0f, 1200.0f, 0.75f, 1.0f, 2.0f, 0.45f, 1.0f, 0.0f,
                            1.0f, 1.0f, 1.0f, 1.0f, 4.0f, 0.35f, 9.0f, 3.0f, 2.0f, 1.2f, 0.25f,
                            0.45f, 5.0f, 4.0f, 3.0f, 0.2f, 40.0f, 1.0f, 1.0f, 1.0f, 1.0f};
    std::memcpy(&s->disk, disk, sizeof disk);
    // GpuCameraPushConstants' defaults (gpu_types.hpp:990-1041)
    s->disk_temperature_scale_k = 23796.0;
    s->disk_temperature_floor_k = 1200.0;
    s->disk_color_saturation = 1.0;
    s->disk_doppler_beaming_exponent = 5.32;
    s->time = 0.0;
    s->camera_exposure = 0.0;
    s->tonemapping_mode = 0;
    s->hydro_model = 0;
    s->accretion_rate_scale = 1.0f;
    s->sky_enabled = 0;
    rt_sky_profile_defaults(&s->sky);
    // GpuHydroDiskProfile's torus defaults (gpu_types.hpp:91-98)
    s->torus_inner_radius = 6.0f;
    s->torus_center_radius = 12.0f;
    s->adiabatic_index = 1.3333334f;
    s->optical_depth_scale = 0.35f;
    s->sampling_density = 2.0f;
}

void rt_sky_profile_defaults(rt_sky_profile* p) {
    if (!p) return;
    const SkyProfile d{};
    std::memcpy(p, &d, sizeof d);
}

namespace {
// Address and type of a sky-profile field by its GpuSkyProfile name: a scalar,
// "name[k]" of a three-float vector, or "grid_cell_colors[c][k]".
void* sky_field(SkyProfile& p, const char* field, int& kind) {
    if (!field) return nullptr;
#define RT_SKY_FIND(T, N, D)                       \
    if (std::strcmp(field, #N) == 0) {             \
        kind = (sizeof(T) == 8) ? 1 : 0;           \
        return &p.N;                               \
    }
    RT_SKY_U32_FIELDS(RT_SKY_FIND)
    RT_SKY_F64_FIELDS(RT_SKY_FIND)
#undef RT_SKY_FIND
    kind = 2;
    const char* br = std::strchr(field, '[');
    if (!br) return nullptr;
    const std::string name(field, br);
    unsigned a = 0, b = 0;
    char tail = 0;
    if (name == "grid_cell_colors") {
        if (std::sscanf(br, "[%u][%u]%c", &a, &b, &tail) != 2 || a >= 16 || b >= 3) return nullptr;
        return &p.grid_cell_colors[a][b];
    }
    if (std::sscanf(br, "[%u]%c", &a, &tail) != 1 || a >= 3) return nullptr;
#define RT_SKY_FINDV(N, A, B, C) \
    if (name == #N) return &p.N[a];
    RT_SKY_VEC_FIELDS(RT_SKY_FINDV)
#undef RT_SKY_FINDV
    return nullptr;
}
}  // namespace

rt_status rt_sky_profile_set(rt_sky_profile* p, const char* field, double value) {
    if (!p) return RT_ERR_INVALID_ARG;
    SkyProfile s;
    std::memcpy(&s, p, sizeof s);
    int kind = 0;
    void* f = sky_field(s, field, kind);
    if (!f) return RT_ERR_INVALID_ARG;
    if (kind == 0) {
        if (!(value >= 0.0 && value <= 4294967295.0)) return RT_ERR_INVALID_ARG;
        *static_cast<uint32_t*>(f) = static_cast<uint32_t>(value);
    } else if (kind == 1) {
        *static_cast<double*>(f) = value;
    } else {
        *static_cast<float*>(f) = static_cast<float>(value);
    }
    std::memcpy(p, &s, sizeof s);
    return RT_OK;
}

rt_status rt_sky_profile_get(const rt_sky_profile* p, const char* field, double* value) {
    if (!p || !value) return RT_ERR_INVALID_ARG;
    SkyProfile s;
    std::memcpy(&s, p, sizeof s);
    int kind = 0;
    const void* f = sky_field(s, field, kind);
    if (!f) return RT_ERR_INVALID_ARG;
    *value = (kind == 0) ? static_cast<double>(*static_cast<const uint32_t*>(f))
             : (kind == 1) ? *static_cast<const double*>(f)
                           : static_cast<double>(*static_cast<const float*>(f));
    return RT_OK;
}

rt_status rt_set_shading(rt_handle* h, const rt_shading* s) {
    if (!h) return RT_ERR_INVALID_ARG;
    if (!s) {
        h->shade_on = false;
        return RT_OK;
    }
    rt_camera probe;
    rt_camera_defaults(&probe);
    ShadeDesc d;
    if (!build_shade_desc(probe, *s, d))
        return fail(h, RT_ERR_INVALID_ARG, "shading: hydro_model 0..2, tonemapping_mode 0..3, sky_enabled 0 or 1");
    h->shading = *s;
    h->shade_on = true;
    return RT_OK;
}

rt_status rt_dispatch(rt_handle* h, const rt_camera* cam, rt_pixel_out* pixels, const rt_ray_out* rays,
                      size_t capacity, const volatile int* cancel) {
    if (!h) return RT_ERR_INVALID_ARG;
    if (!h->ready) return fail(h, RT_ERR_NOT_READY, "handle not ready");
    if (!camera_valid(cam)) return fail(h, RT_ERR_INVALID_ARG, "invalid camera");
    uint32_t row0, nrows;
    row_window(*cam, row0, nrows);
    if (nrows == 0) return fail(h, RT_ERR_INVALID_ARG, "empty row window");
    RT_CUDA(h, cudaSetDevice(h->device));
    if (volume_shading(h, pixels != nullptr)) {
        const rt_camera vc = volume_camera(*cam);
        return dispatch_window(h, &vc, 0, vc.screen_width, row0, nrows, pixels, rays, capacity, cancel);
    }
    return dispatch_window(h, cam, 0, cam->screen_width, row0, nrows, pixels, rays, capacity, cancel);
}

rt_status rt_dispatch_tile(rt_handle* h, const rt_camera* cam, rt_pixel_out* pixels, const rt_ray_out* rays,
                           size_t capacity) {
    if (!h) return RT_ERR_INVALID_ARG;
    if (!h->ready) return fail(h, RT_ERR_NOT_READY, "handle not ready");
    if (!camera_valid(cam)) return fail(h, RT_ERR_INVALID_ARG, "invalid camera");
    // vulkan_compute_executor.hpp:1377-1385
    if (cam->tile_extent_x == 0 || cam->tile_extent_y == 0) return fail(h, RT_ERR_INVALID_ARG, "empty tile");
    if (cam->tile_origin_x >= cam->screen_width || cam->tile_origin_y >= cam->screen_height)
        return fail(h, RT_ERR_INVALID_ARG, "tile origin outside the image");
    const uint32_t w = std::min(cam->tile_extent_x, cam->screen_width - cam->tile_origin_x);
    const uint32_t hgt = std::min(cam->tile_extent_y, cam->screen_height - cam->tile_origin_y);
    RT_CUDA(h, cudaSetDevice(h->device));
    if (volume_shading(h, pixels != nullptr)) {
        const rt_camera vc = volume_camera(*cam);
        return dispatch_window(h, &vc, vc.tile_origin_x, w, vc.tile_origin_y, hgt, pixels, rays, capacity, nullptr);
    }
    return dispatch_window(h, cam, cam->tile_origin_x, w, cam->tile_origin_y, hgt, pixels, rays, capacity, nullptr);
}

rt_status rt_dispatch_device(rt_handle* h, const rt_camera* cam, rt_pixel_out* pixels, const rt_ray_out* rays,
                             size_t capacity, void* stream) {
    if (!h) return RT_ERR_INVALID_ARG;
    if (!h->ready) return fail(h, RT_ERR_NOT_READY, "handle not ready");
    if (!camera_valid(cam)) return fail(h, RT_ERR_INVALID_ARG, "invalid camera");
    if (pixels && (reinterpret_cast<uintptr_t>(pixels) & 15u)) return fail(h, RT_ERR_INVALID_ARG, "pixels not 16-byte aligned");
    uint32_t row0, nrows;
    row_window(*cam, row0, nrows);
    const uint64_t n = static_cast<uint64_t>(cam->screen_width) * nrows;
    if (n == 0) return fail(h, RT_ERR_INVALID_ARG, "empty row window");
    if (capacity < n) return fail(h, RT_ERR_INVALID_ARG, "capacity smaller than the window");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    RT_CUDA(h, cudaSetDevice(h->device));
    rt_camera vc;
    if (volume_shading(h, pixels != nullptr)) {
        vc = volume_camera(*cam);
        cam = &vc;
    }
    rt_ray_out dev = rays ? *rays : rt_ray_out{};
    const bool shade = h->shade_on && pixels;
    rt_status st;
    ContinuationScope cont_scope{h};
    if (shade && (st = add_shade_fields(h, dev, n)) != RT_OK) return st;
    if (is_bl(cam)) {
        // shaded: the shading constants go up before the trace, which follows each
        // ray through the translucent disk
        if (shade && (st = shade_prepare(h, cam, s)) != RT_OK) return st;
        if (shade && (st = begin_continuation(h, n, false, false, s)) != RT_OK) return st;
        if ((st = bl_launch(h, cam, 0, cam->screen_width, row0, nrows, 0, OutPtrs{pixels, dev}, s)) != RT_OK) return st;
        return shade ? shade_launch(h, cam, dev, pixels, n, s, true) : RT_OK;
    }
    if ((st = ensure_host_bundles(h, 1)) != RT_OK) return st;
    if ((st = ensure(h, h->bundles, sizeof(BundleDesc))) != RT_OK) return st;
    // the staging buffer is reused by the next call: wait for the previous upload
    RT_CUDA(h, cudaStreamSynchronize(s));
    build_bundle(*cam, 0, cam->screen_width, row0, nrows, 0, 0, h->host_bundles[0]);
    RT_CUDA(h, cudaMemcpyAsync(h->bundles.ptr, h->host_bundles, sizeof(BundleDesc), cudaMemcpyHostToDevice, s));
    // shaded: the shading constants go up before the trace, which follows each
    // ray through the translucent disk
    if (shade && (st = shade_prepare(h, cam, s)) != RT_OK) return st;
    if (shade && (st = begin_continuation(h, n, false, true, s)) != RT_OK) return st;
    if ((st = launch(h, 1, n, OutPtrs{pixels, dev}, cam->precision_mode == RT_PRECISION_MIXED, s)) != RT_OK) return st;
    return shade ? shade_launch(h, cam, dev, pixels, n, s, true) : RT_OK;
}

uint64_t rt_bundle_rays(const rt_camera* cams, uint32_t n) {
    uint64_t total = 0;
    for (uint32_t b = 0; cams && b < n; ++b) {
        uint32_t row0, nrows;
        row_window(cams[b], row0, nrows);
        total += static_cast<uint64_t>(cams[b].screen_width) * nrows;
    }
    return total;
}

rt_status rt_trace_bundles_device(rt_handle* h, const rt_camera* cams, uint32_t n_bundles, const uint64_t* offsets,
                                  rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity, void* stream) {
    if (!h) return RT_ERR_INVALID_ARG;
    if (!h->ready) return fail(h, RT_ERR_NOT_READY, "handle not ready");
    if (!cams || n_bundles == 0) return fail(h, RT_ERR_INVALID_ARG, "no bundles");
    if (pixels && (reinterpret_cast<uintptr_t>(pixels) & 15u)) return fail(h, RT_ERR_INVALID_ARG, "pixels not 16-byte aligned");
    bool mixed = cams[0].precision_mode == RT_PRECISION_MIXED;
    for (uint32_t b = 0; b < n_bundles; ++b) {
        if (!camera_valid(&cams[b])) return fail(h, RT_ERR_INVALID_ARG, "invalid camera in bundle table");
        if (is_bl(&cams[b]))
            return fail(h, RT_ERR_INVALID_ARG, "Boyer-Lindquist cameras trace through rt_dispatch* (not bundles)");
        if ((cams[b].precision_mode == RT_PRECISION_MIXED) != mixed)
            return fail(h, RT_ERR_INVALID_ARG, "one precision mode per bundle launch");
    }
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    RT_CUDA(h, cudaSetDevice(h->device));
    rt_status st = ensure_host_bundles(h, n_bundles);
    if (st != RT_OK) return st;
    if ((st = ensure(h, h->bundles, sizeof(BundleDesc) * n_bundles)) != RT_OK) return st;
    RT_CUDA(h, cudaStreamSynchronize(s));
    uint64_t begin = 0;
    for (uint32_t b = 0; b < n_bundles; ++b) {
        uint32_t row0, nrows;
        row_window(cams[b], row0, nrows);
        const uint64_t n = static_cast<uint64_t>(cams[b].screen_width) * nrows;
        const uint64_t off = offsets ? offsets[b] : begin;
        if (off + n > capacity) return fail(h, RT_ERR_INVALID_ARG, "bundle outputs exceed capacity");
        build_bundle(cams[b], 0, cams[b].screen_width, row0, nrows, begin, off, h->host_bundles[b]);
        begin += n;
    }
    if (begin == 0) return fail(h, RT_ERR_INVALID_ARG, "empty bundle table");
    OutPtrs out{pixels, rays ? *rays : rt_ray_out{}};
    const rt_launch_config c = effective_cfg(h, mixed);
    if (uses_two_pass(c, mixed, begin) && (st = ensure_two_pass(h, begin)) != RT_OK) return st;
    const bool same = h->graph && h->graph_n_bundles == n_bundles && h->graph_total == begin &&
                      std::memcmp(&h->graph_out, &out, sizeof out) == 0 &&
                      std::memcmp(&h->graph_cfg, &c, sizeof c) == 0;
    if (!same) {
        if (h->graph) cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
        cudaGraph_t g = nullptr;
        RT_CUDA(h, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = cudaMemcpyAsync(h->bundles.ptr, h->host_bundles, sizeof(BundleDesc) * n_bundles,
                                         cudaMemcpyHostToDevice, s);
        rt_status ls = (e1 == cudaSuccess) ? launch(h, n_bundles, begin, out, mixed, s, true) : RT_ERR_DEVICE;
        cudaError_t e2 = cudaStreamEndCapture(s, &g);
        if (e1 != cudaSuccess) return cuda_fail(h, e1, "capture memcpy");
        if (ls != RT_OK) {
            if (g) cudaGraphDestroy(g);
            return ls;
        }
        if (e2 != cudaSuccess) return cuda_fail(h, e2, "cudaStreamEndCapture");
        cudaError_t e3 = cudaGraphInstantiate(&h->graph, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) return cuda_fail(h, e3, "cudaGraphInstantiate");
        h->graph_n_bundles = n_bundles;
        h->graph_total = begin;
        h->graph_out = out;
        h->graph_cfg = c;
    }
    RT_CUDA(h, cudaEventRecord(h->ev0, s));
    RT_CUDA(h, cudaGraphLaunch(h->graph, s));
    RT_CUDA(h, cudaEventRecord(h->ev1, s));
    h->timed = true;
    return RT_OK;
}

rt_status rt_set_launch_config(rt_handle* h, const rt_launch_config* cfg) {
    if (!h || !cfg) return RT_ERR_INVALID_ARG;
    if (cfg->block_size != 0 && cfg->block_size != 64 && cfg->block_size != 128 && cfg->block_size != 256)
        return fail(h, RT_ERR_INVALID_ARG, "block_size must be 64, 128 or 256");
    if (cfg->refill_threshold > 32) return fail(h, RT_ERR_INVALID_ARG, "refill_threshold must be <= 32");
    if (cfg->rays_per_thread > 64) return fail(h, RT_ERR_INVALID_ARG, "rays_per_thread must be <= 64");
    h->cfg = *cfg;
    return RT_OK;
}

rt_status rt_get_launch_config(const rt_handle* h, rt_launch_config* cfg) {
    if (!h || !cfg) return RT_ERR_INVALID_ARG;
    *cfg = effective_cfg(h, false);
    return RT_OK;
}

rt_status rt_synchronize(rt_handle* h, double timeout_ms) {
    if (!h) return RT_ERR_INVALID_ARG;
    return wait_stream(h, h->stream, timeout_ms);
}

rt_status rt_get_stats(rt_handle* h, rt_stats* out) {
    if (!h || !out) return RT_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof *out);
    RT_CUDA(h, cudaSetDevice(h->device));
    RT_CUDA(h, cudaEventSynchronize(h->ev1));
    unsigned long long v[ST_COUNT] = {};
    RT_CUDA(h, cudaMemcpy(v, h->stats.ptr, sizeof v, cudaMemcpyDeviceToHost));
    out->rays = v[ST_RAYS];
    out->attempts = v[ST_ATTEMPTS];
    out->accepted = v[ST_ACCEPTED];
    out->rhs_evals = v[ST_RHS];
    out->fp64_attempts = v[ST_FP64_ATTEMPTS];
    float ms = 0.0f;
    if (h->timed) RT_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    out->kernel_ms = ms;
    return RT_OK;
}

rt_status rt_measure_fma_peak(rt_handle* h, double* fp64_tflops, double* fp32_tflops) {
    if (!h) return RT_ERR_INVALID_ARG;
    RT_CUDA(h, cudaSetDevice(h->device));
    float ms = 0.0f;
    const double f64 = measure_fma_peak(true, h->sm_count, h->stream, &ms);
    const double f32 = measure_fma_peak(false, h->sm_count, h->stream, &ms);
    RT_CUDA(h, cudaGetLastError());
    if (fp64_tflops) *fp64_tflops = f64;
    if (fp32_tflops) *fp32_tflops = f32;
    return RT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free bundle trace (rt_trace_bundles_noalloc).
//
// The scratch of the persistent launch (ray-queue counter, launch counters,
// bundle table) lives in one static device array per device instead of
// handle-owned cudaMalloc buffers; the kernel is the same one the handle
// entry points launch.

namespace {

constexpr size_t kNoAllocCounterBytes = 256;  // queue counter at byte 0, launch counters at byte 64
constexpr size_t kNoAllocStatsOffset = 64;
constexpr size_t kNoAllocScratchBytes = kNoAllocCounterBytes + RT_NOALLOC_MAX_BUNDLES * sizeof(BundleDesc);
static_assert(kNoAllocScratchBytes == RT_NOALLOC_SCRATCH_BYTES, "header states the scratch size");
static_assert(kNoAllocStatsOffset + ST_COUNT * sizeof(unsigned long long) <= kNoAllocCounterBytes,
              "launch counters fit the zeroed block");

}  // namespace

// Bytes [0, 256): counters, zeroed by every call; bytes [256, ...): bundle table.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;

struct NoAllocDevice {
    unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int sm_count = 0;
};

// Puts the caller's current device back when the entry point returns.
struct DeviceRestore {
    int prev = -1;
    ~DeviceRestore() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

std::mutex g_noalloc_mutex;
NoAllocDevice g_noalloc_devices[kNoAllocMaxDevices];

rt_status noalloc_fail(char* buf, size_t len, rt_status st, const char* msg, const char* detail = nullptr) {
    if (buf && len > 0) std::snprintf(buf, len, "%s%s%s", msg, detail ? ": " : "", detail ? detail : "");
    return st;
}

rt_status noalloc_cuda_fail(char* buf, size_t len, cudaError_t e, const char* where) {
    cudaGetLastError();
    return noalloc_fail(buf, len, e == cudaErrorMemoryAllocation ? RT_ERR_OOM : RT_ERR_DEVICE, where,
                        cudaGetErrorString(e));
}

// Per-device set-up, once: device check, scratch address, kernel loading.
// The caller has made `dev` current.
rt_status noalloc_setup(int dev, NoAllocDevice& out, char* err, size_t len) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocDevice& d = g_noalloc_devices[dev];
    if (!d.scratch) {
        int major = 0, minor = 0, sms = 0;
        cudaError_t e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return noalloc_cuda_fail(err, len, e, "cudaDeviceGetAttribute");
        if (major != 10 || minor != 0) return noalloc_fail(err, len, RT_ERR_DEVICE, "device is not sm_100");
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return noalloc_cuda_fail(err, len, e, "cudaGetSymbolAddress");
        // load every tracer kernel now (occupancy queries load them), not inside a later call
        for (uint32_t block : {64u, 128u, 256u})
            for (bool mixed : {false, true})
                for (bool rolled : {false, true}) trace_occupancy(kernel_block(block, mixed, rolled), mixed, rolled);
        if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_cuda_fail(err, len, e, "kernel set-up");
        d.scratch = static_cast<unsigned char*>(p);
        d.sm_count = sms;
    }
    out = d;
    return RT_OK;
}

}  // namespace

extern "C" rt_status rt_trace_bundles_noalloc(int device_ordinal, const rt_camera* cams, uint32_t n_bundles,
                                              const uint64_t* offsets, rt_pixel_out* pixels, const rt_ray_out* rays,
                                              size_t capacity, const rt_launch_config* cfg, void* stream,
                                              char* error, size_t error_len) {
    if (error && error_len > 0) error[0] = '\0';
    if (!cams || n_bundles == 0) return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "no bundles");
    if (n_bundles > RT_NOALLOC_MAX_BUNDLES) {
        char detail[96];
        std::snprintf(detail, sizeof detail, "%u bundles requested, the static scratch holds at most %d",
                      n_bundles, RT_NOALLOC_MAX_BUNDLES);
        return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "bundle table too long", detail);
    }
    if (pixels && (reinterpret_cast<uintptr_t>(pixels) & 15u))
        return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "pixels not 16-byte aligned");
    if (cfg && ((cfg->block_size != 0 && cfg->block_size != 64 && cfg->block_size != 128 && cfg->block_size != 256) ||
                cfg->refill_threshold > 32 || cfg->rays_per_thread > 64))
        return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "invalid launch config");
    const bool mixed = cams[0].precision_mode == RT_PRECISION_MIXED;
    for (uint32_t b = 0; b < n_bundles; ++b) {
        if (!camera_valid(&cams[b]))
            return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "invalid camera in bundle table");
        if (is_bl(&cams[b]))
            return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "Boyer-Lindquist cameras are not bundle cameras");
        if ((cams[b].precision_mode == RT_PRECISION_MIXED) != mixed)
            return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "one precision mode per bundle launch");
    }
    // bundle table on the host stack
    BundleDesc table[RT_NOALLOC_MAX_BUNDLES];
    uint64_t begin = 0;
    for (uint32_t b = 0; b < n_bundles; ++b) {
        uint32_t row0, nrows;
        row_window(cams[b], row0, nrows);
        const uint64_t n = static_cast<uint64_t>(cams[b].screen_width) * nrows;
        const uint64_t off = offsets ? offsets[b] : begin;
        if (off + n > capacity)
            return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "bundle outputs exceed capacity");
        build_bundle(cams[b], 0, cams[b].screen_width, row0, nrows, begin, off, table[b]);
        begin += n;
    }
    if (begin == 0) return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "empty bundle table");

    int n_dev = 0;
    cudaError_t e = cudaGetDeviceCount(&n_dev);
    if (e != cudaSuccess) return noalloc_cuda_fail(error, error_len, e, "cudaGetDeviceCount");
    if (device_ordinal < 0 || device_ordinal >= n_dev || device_ordinal >= kNoAllocMaxDevices)
        return noalloc_fail(error, error_len, RT_ERR_DEVICE, "no such device");
    // the caller's current device is put back on every return path
    DeviceRestore restore;
    if ((e = cudaGetDevice(&restore.prev)) != cudaSuccess) return noalloc_cuda_fail(error, error_len, e, "cudaGetDevice");
    if ((e = cudaSetDevice(device_ordinal)) != cudaSuccess) return noalloc_cuda_fail(error, error_len, e, "cudaSetDevice");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the bundle table is uploaded from this call's stack frame, which a graph
    // replay could not read again: refuse capture before anything is enqueued
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(s, &capture)) != cudaSuccess)
        return noalloc_cuda_fail(error, error_len, e, "stream capture check");
    if (capture != cudaStreamCaptureStatusNone)
        return noalloc_fail(error, error_len, RT_ERR_INVALID_ARG, "stream is capturing",
                            "the allocation-free call cannot be captured into a CUDA graph");
    NoAllocDevice dev;
    rt_status st = noalloc_setup(device_ordinal, dev, error, error_len);
    if (st != RT_OK) return st;

    // effective_cfg reads only the handle's launch config
    rt_handle shape;
    if (cfg) shape.cfg = *cfg;
    const rt_launch_config c = effective_cfg(&shape, mixed);

    unsigned char* table_dev = dev.scratch + kNoAllocCounterBytes;
    // pageable source: the copy is staged before the call returns, after the stream's earlier work
    if ((e = cudaMemcpyAsync(table_dev, table, sizeof(BundleDesc) * n_bundles, cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
        return noalloc_cuda_fail(error, error_len, e, "bundle table upload");
    if ((e = cudaMemsetAsync(dev.scratch, 0, kNoAllocCounterBytes, s)) != cudaSuccess)
        return noalloc_cuda_fail(error, error_len, e, "counter reset");
    TraceArgs args{};
    args.bundles = reinterpret_cast<const BundleDesc*>(table_dev);
    args.n_bundles = n_bundles;
    args.refill_threshold = c.refill_threshold;
    args.claim = 32u * c.rays_per_thread;
    args.total_rays = begin;
    args.queue = reinterpret_cast<unsigned long long*>(dev.scratch);
    args.stats = reinterpret_cast<unsigned long long*>(dev.scratch + kNoAllocStatsOffset);
    args.out = OutPtrs{pixels, rays ? *rays : rt_ray_out{}};
    const uint32_t grid = static_cast<uint32_t>(dev.sm_count) * c.ctas_per_sm;
    launch_trace(args, grid, c.block_size, mixed, c.fp64_rolled != 0, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_cuda_fail(error, error_len, e, "tracer launch");
    return RT_OK;
}
