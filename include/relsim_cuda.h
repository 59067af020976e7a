/*
 * relsim_cuda.h -- C ABI of the B200 (sm_100a) backward null-geodesic tracer.
 *
 * Drop-in compute backend for Wartets/Relativity-Simulator's image path.  Each
 * entry point names the reference interface it replaces (paths relative to the
 * reference source tree):
 *
 *   rt_create / rt_destroy     VulkanComputeExecutor::initialize / shutdown
 *                              (include/relativistic/render/vulkan_compute_executor.hpp:983-987, 1272)
 *   rt_is_ready                VulkanComputeExecutor::is_ready (:1257)
 *   rt_is_platform_supported   VulkanComputeExecutor::is_platform_supported (:1634)
 *   rt_dispatch                VulkanComputeExecutor::dispatch_and_readback (:1399-1464)
 *   rt_dispatch_tile           VulkanComputeExecutor::dispatch_tile_and_readback (:1372-1391)
 *   rt_camera                  hot-path subset of GpuCameraPushConstants
 *                              (include/relativistic/render/gpu_types.hpp:966-1109)
 *   rt_pixel_out               GpuPixelOutput, same 32-byte layout (gpu_types.hpp:1111-1121)
 *   RT_PIXEL_*                 PixelFlags (gpu_types.hpp:1123-1130)
 *
 * Beyond the reference: a per-ray SoA record (class, final BL position, disk
 * radius, redshift, invariant drift), device-resident dispatch, batched camera
 * bundles in one persistent launch, and a continuous-batching request server.
 *
 * Conventions: every call returns rt_status, never throws; host buffers are
 * caller-owned; device buffers are owned by the handle and grow on demand.  A
 * handle is thread-compatible (one CUDA stream per handle): callers serialise
 * calls on one handle, as the reference's pipeline does with gpu_mutex_.
 * There is no CPU fallback inside this library; a missing or failed device
 * is reported as RT_ERR_DEVICE / RT_ERR_NOT_READY.
 */
#ifndef RELSIM_CUDA_H
#define RELSIM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RT_ABI_VERSION 5

typedef enum rt_status {
    RT_OK = 0,
    RT_ERR_INVALID_ARG = 1,
    RT_ERR_OOM = 2,
    RT_ERR_TIMEOUT = 3,
    RT_ERR_DEVICE = 4,
    RT_ERR_CANCELLED = 5,
    RT_ERR_NOT_READY = 6,
    RT_ERR_BUDGET = 7,   /* request larger than the device-memory budget */
    RT_ERR_AGAIN = 8     /* server queue full; retry after rt_server_poll */
} rt_status;

typedef enum rt_precision {
    RT_PRECISION_FP64 = 0,  /* every stage in FP64 (the plain tracer) */
    RT_PRECISION_MIXED = 1  /* FP32 far-field stages, FP64 state / near zone */
} rt_precision;

/* Ray classes written to rt_ray_out.status. */
enum {
    RT_RAY_UNFINISHED = 0,  /* step budget exhausted */
    RT_RAY_CAPTURED = 1,    /* r_BL < capture_scale * r_+, or non-finite state */
    RT_RAY_ESCAPED = 2,     /* r_BL > escape_radius */
    RT_RAY_DISK = 3         /* first z = 0 crossing with r in [r_in, r_out] */
};
/* Ray flags written to rt_ray_out.flags. */
enum {
    RT_RAYFLAG_NONFINITE = 1u << 0,
    RT_RAYFLAG_STEP_UNDERFLOW = 1u << 1,
    RT_RAYFLAG_MAX_STEPS = 1u << 2,
    RT_RAYFLAG_EARLY_CAPTURE = 1u << 3
    /* bit 4: RT_RAYFLAG_DIVERGED (multi-source, below) */
};
/* PixelFlags (gpu_types.hpp:1123-1130). */
#define RT_PIXEL_HORIZON_ABSORBED (1u << 0)
#define RT_PIXEL_CELESTIAL_HIT (1u << 1)
#define RT_PIXEL_ACCRETION_DISK_HIT (1u << 2)

/* Coordinate form of the traced metric (rt_camera.metric_form). */
typedef enum rt_metric_form {
    /* Kerr: Kerr-Schild Hamiltonian tracer (metric types 2 and 3 of the
     * reference, trace_kerr_schild_photon, software_compute_engine.hpp:3370) */
    RT_METRIC_KERR_SCHILD = 0,
    /* Kerr-Newman in Boyer-Lindquist coordinates with charge metric_charge:
     * geodesic equation -Gamma u u from the ZAMO ray (metric type 5,
     * KerrNewmanMetric; with charge 0 the KerrMetric default route; with
     * spin and charge 0 Schwarzschild, metric type 1) -- trace_exact_photon,
     * software_compute_engine.hpp:1334-1622, routed at :3364-3391.  FP64
     * always (precision_mode is not used); a^2 + Q^2 < M^2 required. */
    RT_METRIC_BOYER_LINDQUIST = 1
} rt_metric_form;

/* Camera and integration parameters of one image (one "bundle"). */
typedef struct rt_camera {
    double observer_position[4]; /* t, r, theta, phi (Boyer-Lindquist), as GpuCameraPushConstants */
    double tetrad_e1[4];         /* forward; spatial part in [1..3] */
    double tetrad_e2[4];         /* right */
    double tetrad_e3[4];         /* up */
    double field_of_view_rad;
    double metric_mass;          /* clamped to >= 1e-4 */
    double metric_spin;          /* clamped to |a| <= 0.999 M (software_compute_engine.hpp:3801) */
    double escape_radius;
    double capture_scale;        /* captured when r_BL < capture_scale * r_+ */
    double disk_inner_radius;    /* <= 0: r_ISCO(a) */
    double disk_outer_radius;    /* <= 0: no disk */
    double rtol;                 /* DP45 relative tolerance */
    double atol;                 /* DP45 absolute tolerance */
    double step_cap_fraction;    /* |h| <= c * max(r_BL - r_+, 0.01 M) */
    double initial_step_fraction;/* |h0| = f * r_obs */
    double projection_tol;       /* project onto H = 0 when |H| >= tol */
    double mixed_fp64_radius;    /* MIXED: FP64 stages inside this r_BL (<= 0: max(3 r_+, 5 M)) */
    double metric_charge;        /* Q (G = c = k_e = 1), RT_METRIC_BOYER_LINDQUIST only */
    double mixed_critical_band;  /* MIXED: a ray whose constants lie within this distance (M, in impact
                                    parameter) of the critical curve orbits the photon region, where step
                                    errors grow about as 1/distance; it is traced in FP64 at a hundredth of
                                    rtol and atol from its first step (0: 1 M; < 0: none) */
    uint32_t screen_width;
    uint32_t screen_height;
    uint32_t max_integration_steps; /* step attempts per ray, accepted + rejected */
    uint32_t early_capture;      /* 1: end a ray once capture is certain */
    uint32_t precision_mode;     /* rt_precision */
    uint32_t dispatch_row_offset;/* row window as GpuCameraPushConstants; count 0 = all rows */
    uint32_t dispatch_row_count;
    uint32_t tile_origin_x;      /* tile window for rt_dispatch_tile */
    uint32_t tile_origin_y;
    uint32_t tile_extent_x;
    uint32_t tile_extent_y;
    uint32_t metric_form;        /* rt_metric_form */
} rt_camera;

/* GpuPixelOutput (gpu_types.hpp:1111-1121): 32 bytes. */
typedef struct rt_pixel_out {
    float r, g, b, a;
    float redshift;
    float affine_parameter;
    uint32_t status_flags;
    uint32_t iterations_used;
} rt_pixel_out;

/* GpuDiskProfile (gpu_types.hpp:42-78): the disk's appearance, 32 floats in
 * the reference's order (a GpuDiskProfile can be copied in directly). */
typedef struct rt_disk_profile {
    float enabled, inner_radius_scale, outer_radius_mass_units, peak_temperature_k;
    float floor_temperature_k, temperature_exponent, zero_torque_strength, extra_beaming_exponent;
    float brightness, color_saturation, tint_strength, opacity_scale;
    float tint_r, tint_g, tint_b, rotation_speed_scale;
    float ring_amplitude, ring_frequency, ring_sharpness, spiral_arm_count;
    float spiral_pitch, spiral_amplitude, turbulence_amplitude, turbulence_scale;
    float turbulence_octaves, radial_stretch, grain_amplitude, grain_scale;
    float reference_luminance, noise_seed, temperature_normalization, edge_softness;
} rt_disk_profile;

/* Pixel shading of GpuPixelOutput's colour (the reference's shading tail,
 * software_compute_engine.hpp:1538-1611, 1734-1808): each disk crossing is
 * shaded as the thin disk at (r, phi, g) -- temperature profile, rings,
 * spiral arms, turbulence, blackbody colour, Doppler beaming, grading -- and
 * the disk is translucent, as in the reference: a crossing adds its radiance
 * at the throughput left and lowers the throughput by its opacity, and the
 * ray is followed on while more than 0.01 is left (the per-ray record still
 * describes the first hit; a disk pixel's flags add how the ray ended and its
 * redshift is the last crossing's).  A ray that escapes, or ends with more
 * than 0.01 of its throughput outside 3 r_s, adds the procedural sky
 * (SkyboxRenderer, render/skybox_renderer.hpp) at its exit direction times
 * the throughput left when sky_enabled is 1 (software_compute_engine.hpp:
 * 1766-1795).  The sum is tonemapped to sRGB.  Fields as in
 * GpuCameraPushConstants (gpu_types.hpp:990-1106); the disk profile is
 * resolved as AccretionDiskModel::resolve_primary_profile does. */
/* The procedural sky's settings: the byte image of GpuSkyProfile
 * (gpu_types.hpp:273-964), so a GpuSkyProfile copies in directly.
 * rt_sky_profile_defaults gives its defaults; rt_sky_profile_set / _get read
 * and write a field by its GpuSkyProfile name ("star_density", "seed",
 * "nebula_emission_color[1]", "grid_cell_colors[3][0]"). */
typedef struct rt_sky_profile {
    unsigned char bytes[1808];
} rt_sky_profile;
typedef struct rt_shading {
    rt_disk_profile disk;                 /* primary_disk */
    double disk_temperature_scale_k;      /* overrides disk.peak_temperature_k */
    double disk_temperature_floor_k;      /* overrides disk.floor_temperature_k */
    double disk_color_saturation;         /* overrides disk.color_saturation */
    double disk_doppler_beaming_exponent; /* overrides disk.extra_beaming_exponent */
    double time;                          /* animation time of the disk pattern and the sky */
    double camera_exposure;               /* EV */
    uint32_t tonemapping_mode;            /* 0 clamp, 1 ACES fit, 2 log luminance, 3 extended Reinhard */
    uint32_t hydro_model;                 /* hydro_disk.model: 0 procedural profile, 1 Novikov-Thorne flux,
                                             2 Fishbone-Moncrief torus */
    float accretion_rate_scale;           /* hydro_disk.accretion_rate_scale (Novikov-Thorne) */
    uint32_t sky_enabled;                 /* 1: the procedural sky behind escaped rays (sky.enabled
                                             switches it off as well); the reference's image
                                             panoramas (sky_background_source != 0) are not part of
                                             this library */
    rt_sky_profile sky;                   /* sky (GpuSkyProfile) */
    /* hydro model 2, the Fishbone-Moncrief torus (hydro_disk, GpuHydroDiskProfile,
       gpu_types.hpp:91-107): inner edge and pressure maximum in units of M, the
       adiabatic index, the optical depth scale and the samples per M of chord */
    float torus_inner_radius;
    float torus_center_radius;
    float adiabatic_index;
    float optical_depth_scale;
    float sampling_density;
    float reserved_torus;
} rt_shading;

/* Per-ray record, structure of arrays.  Any pointer may be NULL (not written).
 * Pointers are host pointers for rt_dispatch* and device pointers for the
 * *_device entry points. */
typedef struct rt_ray_out {
    uint32_t* status;
    uint32_t* flags;
    uint32_t* steps_accepted;
    uint32_t* steps_rejected;
    double* r;       /* final BL radius */
    double* theta;   /* final BL polar angle */
    double* phi;     /* final azimuth, unwrapped along the ray */
    double* r_hit;   /* disk-hit radius, NaN without a hit */
    double* g;       /* disk redshift factor, 1 without a hit */
    double* lambda;  /* affine parameter at termination (negative: traced backwards) */
    double* dH;      /* max |H| before each projection */
    double* dE;      /* -p_t recomputed from the null condition at the end, minus 1 */
    double* dLz;     /* L_z(end) - L_z(start) */
    double* dQ;      /* Carter Q(end) - Q(start) */
    /* escaped rays: unit Cartesian direction (x, y, z) at the escape radius that
     * the reference's sky lookup takes: -dx/dlambda / |dx/dlambda| of the
     * Kerr-Schild state (software_compute_engine.hpp:1771-1775; the superposed
     * flow for multi-source scenes, :3220-3224), or the orthonormal-frame
     * velocity of the Boyer-Lindquist state mapped to a direction of travel
     * (:1581-1589).  NaN for other rays.  Not recorded by the request server. */
    double* exit_x;
    double* exit_y;
    double* exit_z;
    /* the body the ray ended on: for a disk hit the source whose disk it hit
     * first, for a capture the source that captured it (0: the camera's hole,
     * k: the k-th rt_source of a multi-source scene); RT_BODY_NONE for escaped
     * and unfinished rays and for captures in a horizon-like region of the
     * summed fields (RT_RAYFLAG_DIVERGED).  Not recorded by the request server. */
    uint32_t* body;
} rt_ray_out;
#define RT_BODY_NONE 0xFFFFFFFFu

/* Launch shape of the persistent tracer (set by the autotuner). */
typedef struct rt_launch_config {
    uint32_t block_size;       /* threads per CTA: 64, 128, 256 */
    uint32_t ctas_per_sm;      /* persistent CTAs per SM; 0 = occupancy maximum */
    uint32_t refill_threshold; /* idle lanes of a warp before it refills from the queue */
    uint32_t rays_per_thread;  /* consecutive rays claimed per lane with each global atomic:
                                  a warp claims 32 * rays_per_thread rays at a time (1..64) */
    uint32_t fp64_rolled;      /* FP64 mode: 1 = stage loop rolled around one RHS copy with the
                                  stage derivatives in shared memory, 0 = straight-line stages */
    uint32_t mixed_single_kernel; /* MIXED mode: 0 = two passes per round, an FP32 far-zone kernel and
                                  an FP64 near-zone kernel exchanging parked rays through HBM (the
                                  default); 1 = one kernel, FP64 steps for a whole warp whenever one
                                  of its rays is in the FP64 zone (rolled FP64 step) */
} rt_launch_config;

/* Counters of the last dispatch (device-side totals). */
typedef struct rt_stats {
    uint64_t rays;
    uint64_t attempts;       /* DP45 step attempts, accepted + rejected */
    uint64_t accepted;
    uint64_t rhs_evals;
    uint64_t fp64_attempts;  /* attempts taken in FP64 (all of them in FP64 mode) */
    double kernel_ms;        /* device time of the tracer kernel(s) */
} rt_stats;

typedef struct rt_handle rt_handle;

/* Lifetime (VulkanComputeExecutor::initialize / shutdown). */
rt_status rt_create(rt_handle** out, int device_ordinal);
void rt_destroy(rt_handle* h);
int rt_is_ready(const rt_handle* h);
int rt_is_platform_supported(void);
const char* rt_last_error(const rt_handle* h);
int rt_abi_version(void);

/* ---- Multi-source Kerr-Schild superposition ----
 * SoftwareComputeEngine's multi-source path (software_compute_engine.hpp:
 * 2708-3252, trace_multi_source): the camera's hole at the origin plus black-
 * hole bodies (GpuBodyData with preset 8), each with its own mass, spin axis
 * and thin disk; the ray equations sum every source's Kerr-Schild terms in its
 * local frame.  Traced in FP64 with the DP45 machinery of the single-hole
 * tracer: projection onto H = 0 of the superposed Hamiltonian, step cap from
 * the nearest source, captured inside capture_scale * r_+ of any source (or,
 * flag RT_RAYFLAG_DIVERGED, when the momentum exceeds 1000: a horizon-like
 * region of the summed fields), escaped at |x| > escape_radius, disk hit at a
 * source's first equatorial crossing on its disk (g from that source's disk).
 * The record's r, theta, phi are spherical about the origin; dE, dLz, dQ are
 * NaN (no Kerr invariants for the superposition); body names the source of the
 * first disk hit or of the capture.  Shaded (rt_set_shading, pixels
 * requested), every ray is followed through the translucent disks of all
 * sources, each step's crossings in order along the ray, and each crossing is
 * shaded with its source's disk: the camera's hole with rt_shading.disk
 * resolved, a body with rt_source.disk as it stands, both by the thin
 * procedural model at detail 1 (software_compute_engine.hpp:3150-3191); a ray
 * that ends within 6 m of a source with throughput left adds no sky
 * (:3207-3216).  The camera's rtol and atol apply (the mixed mode's 1e-8 for a
 * mixed-mode camera; the stages stay FP64). */
#define RT_MAX_SOURCES 16        /* the camera's hole and up to 15 sources */
#define RT_RAYFLAG_DIVERGED (1u << 4)

/* A black-hole body (GpuBodyData, gpu_types.hpp:1213-1307, preset 8). */
typedef struct rt_source {
    double position[3];
    double mass;
    double spin_parameter;  /* a / m, clamped to [-0.9999, 0.9999] */
    double axis[3];         /* spin axis (normalised here; zero selects +z) */
    double disk_enabled;    /* > 0.5: thin disk */
    double disk_inner_scale;/* inner radius = max(scale, 1) * r_ISCO of the source */
    double disk_outer_units;/* outer radius = max(units * mass, 1.05 * inner) */
    rt_disk_profile disk;   /* the body's disk appearance (GpuBodyData::disk), used as it stands when
                               shading; the camera's hole uses rt_shading.disk */
} rt_source;

/* Trace the row window of a multi-source scene (host buffers, as rt_dispatch).
 * The camera's metric_mass / metric_spin / disk describe the hole at the
 * origin; n_sources <= RT_MAX_SOURCES - 1 more.  FP64 stages. */
rt_status rt_dispatch_multi(rt_handle* h, const rt_camera* cam, const rt_source* sources, uint32_t n_sources,
                            rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity);
/* Device-resident form: device outputs, enqueued on `stream` (NULL: the handle's). */
rt_status rt_dispatch_multi_device(rt_handle* h, const rt_camera* cam, const rt_source* sources, uint32_t n_sources,
                                   rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity, void* stream);

/* Prograde/retrograde ISCO radius by the sign of the spin
 * (SoftwareComputeEngine::kerr_isco_radius, software_compute_engine.hpp:1052-1061). */
double rt_kerr_isco_radius(double mass, double spin);

/* Defaults: r=100, i=17 deg, FOV 12 deg, a=0.94, 2048^2, disk [r_ISCO, 20],
 * rtol=atol=1e-10, cap 0.1, h0 = 0.01 r_obs, 20000 attempts, FP64. */
void rt_camera_defaults(rt_camera* cam);
/* Fill observer_position and the forward/right/up tetrad of a static observer
 * at (r, theta, phi) looking at the hole (forward = -e_r, right = e_phi, up = -e_theta). */
void rt_camera_look_at_hole(rt_camera* cam, double r, double theta, double phi);

/* Trace the row window of the image (VulkanComputeExecutor::dispatch_and_readback).
 * Host buffers; pixels and/or rays may be NULL; capacity = elements available,
 * which must be >= width * rows of the window.  cancel (optional) is polled
 * between bands: a non-zero value returns RT_ERR_CANCELLED. */
rt_status rt_dispatch(rt_handle* h, const rt_camera* cam, rt_pixel_out* pixels, const rt_ray_out* rays,
                      size_t capacity, const volatile int* cancel);

/* Trace the tile [origin, origin + extent) in tile-major order
 * (VulkanComputeExecutor::dispatch_tile_and_readback). */
rt_status rt_dispatch_tile(rt_handle* h, const rt_camera* cam, rt_pixel_out* pixels, const rt_ray_out* rays,
                           size_t capacity);

/* Device-resident form: pixels/rays are device pointers, work is enqueued on
 * `stream` (a cudaStream_t; NULL = the handle's stream) and not waited for. */
rt_status rt_dispatch_device(rt_handle* h, const rt_camera* cam, rt_pixel_out* pixels, const rt_ray_out* rays,
                             size_t capacity, void* stream);

/* Batched camera bundles of uneven size in one persistent launch.  Bundle b's
 * rays are written at offset offsets[b] of the (device) outputs, row-major
 * within the bundle's row window; offsets may be NULL (packed in order).
 * The launch is captured into a CUDA graph and replayed while the bundle
 * table's shape is unchanged. */
rt_status rt_trace_bundles_device(rt_handle* h, const rt_camera* cams, uint32_t n_bundles, const uint64_t* offsets,
                                  rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity, void* stream);

/* Total rays of a bundle table (sum of the row windows). */
uint64_t rt_bundle_rays(const rt_camera* cams, uint32_t n_bundles);

/* Launch configuration (the autotuner writes it; zeros select defaults). */
rt_status rt_set_launch_config(rt_handle* h, const rt_launch_config* cfg);

/* Shade the pixels of later rt_dispatch, rt_dispatch_tile, rt_dispatch_device
 * and rt_dispatch_multi* calls on this handle; NULL turns shading off
 * (r = g = b = 0, a = 1, the default).  RT_ERR_INVALID_ARG for hydro_model
 * above 2, sky_enabled above 1 or tonemapping_mode above 3.  Hydro model 2,
 * the Fishbone-Moncrief torus, shades single-hole cameras: they are traced by
 * an FP64 tracer at the camera's tolerances with no thin disk and no early
 * capture, gathering each step's chord through the torus
 * (software_compute_engine.hpp:1529-1537, 1725-1731), so their records
 * describe that trace.  Multi-source dispatches draw no torus: the camera
 * hole's disk is off and the bodies' disks are shaded as usual, as the
 * reference's multi-source path does (:2752).  rt_server_set_shading refuses
 * hydro_model 2.  rt_shading_defaults
 * gives the reference's defaults for the disk and the tonemap, GpuSkyProfile's
 * defaults in sky, and sky_enabled = 0 (black behind the disk; set it to 1 for
 * the reference's sky). */
void rt_shading_defaults(rt_shading* s);
rt_status rt_set_shading(rt_handle* h, const rt_shading* s);
/* GpuSkyProfile's defaults, and one field by name (see rt_sky_profile):
 * RT_ERR_INVALID_ARG for an unknown name or index. */
void rt_sky_profile_defaults(rt_sky_profile* p);
rt_status rt_sky_profile_set(rt_sky_profile* p, const char* field, double value);
rt_status rt_sky_profile_get(const rt_sky_profile* p, const char* field, double* value);
rt_status rt_get_launch_config(const rt_handle* h, rt_launch_config* cfg);

/* Counters of the last dispatch; waits for it to finish. */
rt_status rt_get_stats(rt_handle* h, rt_stats* stats);

/* Wait for the handle's stream with a wall-clock limit (ms); RT_ERR_TIMEOUT
 * when the limit passes first (the work is not cancelled). */
rt_status rt_synchronize(rt_handle* h, double timeout_ms);

/* Measured FMA throughput of this device (TFLOP/s, an FMA counted as 2 FLOP),
 * from a register-resident FMA-chain kernel.  Roofline denominator. */
rt_status rt_measure_fma_peak(rt_handle* h, double* fp64_tflops, double* fp32_tflops);

/* ---- Continuous-batching request server ----
 * Replaces the reference's frame-at-a-time render worker
 * (GeodesicComputePipeline, geodesic_compute_pipeline.hpp:505-529, which
 * serialises whole frames on one executor under gpu_mutex_) for a stream of
 * render requests.  Requests are admitted in arrival order while their output
 * records fit memory_budget_bytes of device memory, and traced in epochs: one
 * persistent launch over row chunks taken round-robin from every admitted
 * request, so a request arriving while others are on the GPU joins the next
 * epoch.  Records stay on the device until a request's last chunk is done,
 * then go to the caller's host buffers.  Besides the budget, the server holds
 * two epochs' ray state for the two-pass mixed tracer (124 bytes per epoch ray
 * per slot: about 1 GB at the default 2^22-ray epochs).  A scheduler thread owned by the server
 * does all device work; submit and poll may be called from any thread. */
typedef struct rt_server rt_server;

typedef struct rt_server_config {
    uint64_t memory_budget_bytes;  /* device bytes for in-flight output records (admission budget) */
    uint32_t max_requests;         /* waiting + admitted requests; more: RT_ERR_AGAIN */
    uint32_t chunk_rays;           /* cost units a request contributes to one epoch (whole rows) */
    uint32_t epoch_rays;           /* cost units per epoch launch; also its ray capacity.  A ray costs
                                      1 unit (mixed Kerr-Schild), 2 (FP64), 4 (Boyer-Lindquist) or,
                                      multi-source, 2 per hole at rtol >= 1e-9 and 4 below; an epoch's
                                      first chunk takes at least one row */
    uint32_t max_epoch_bundles;    /* row chunks per epoch launch */
    uint32_t record_mask;          /* bit f: rt_ray_out field f (declaration order) is recorded;
                                      bit 14: the 32-byte pixels */
    uint32_t min_epoch_rays;       /* an epoch keeps taking rows up to this many rays even past its
                                      cost units (keeps a launch of slow rays long enough to fill
                                      the GPU); capped at epoch_rays */
    rt_launch_config launch_fp64;  /* launch shapes; zeros select the defaults */
    rt_launch_config launch_mixed;
    uint32_t multi_source_sms;     /* SMs' worth of persistent CTAs a multi-source epoch launches
                                      (0: every SM); fewer leave room for a single-hole epoch on the
                                      other slot to run beside it */
    uint32_t reserved;
} rt_server_config;

typedef struct rt_request_done {
    uint64_t id;
    uint64_t rays;
    double latency_ms;  /* submit to records in the caller's host buffers */
    double queue_ms;    /* submit to the first epoch launch that traces it */
    rt_status status;
    uint32_t reserved;
} rt_request_done;

typedef struct rt_server_stats {
    uint64_t requests_submitted, requests_done, rays_done;
    uint64_t epochs, bundles;                  /* launches and row chunks traced */
    uint64_t bytes_in_use, peak_bytes_in_use;  /* admitted requests' records */
    uint64_t budget_bytes;                     /* usable budget (whole rays) */
    uint32_t pending;                          /* waiting + admitted, not yet polled as done */
    uint32_t peak_active;                      /* most requests admitted at once */
    uint64_t peak_epoch_rays;                  /* most rays in one epoch launch (<= epoch_rays) */
} rt_server_stats;

/* Defaults: 1 GiB budget, 4096 requests, 2^18-unit chunks, 2^22-unit epochs of at
 * least 2^18 rays, records status, r, theta, phi, r_hit, g and the pixels. */
void rt_server_config_defaults(rt_server_config* cfg);
rt_status rt_server_create(rt_server** out, int device_ordinal, const rt_server_config* cfg);
/* Stops the scheduler; requests not yet done are dropped. */
void rt_server_destroy(rt_server* s);
/* Queue one request.  Host buffers (pinned memory overlaps best) must stay valid
 * until the request is polled as done and may only name recorded fields.
 * RT_ERR_AGAIN: max_requests reached; RT_ERR_BUDGET: larger than the whole budget;
 * RT_ERR_INVALID_ARG also for a row wider than epoch_rays. */
rt_status rt_server_submit(rt_server* s, const rt_camera* cam, rt_pixel_out* pixels, const rt_ray_out* rays,
                           size_t capacity, uint64_t* id);
/* Queue a multi-source scene (see rt_dispatch_multi; FP64 stages). */
rt_status rt_server_submit_multi(rt_server* s, const rt_camera* cam, const rt_source* sources, uint32_t n_sources,
                                 rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity, uint64_t* id);
/* Up to max_done finished requests, waiting at most timeout_ms for the first. */
rt_status rt_server_poll(rt_server* s, rt_request_done* done, uint32_t max_done, uint32_t* n_done,
                         double timeout_ms);
rt_status rt_server_get_stats(rt_server* s, rt_server_stats* stats);
const char* rt_server_last_error(const rt_server* s);
/* Shade the pixels of requests that finish from now on (single-hole cameras of
 * both metric forms, at their first disk crossing -- the server's epochs hold
 * no continuation state; multi-source requests keep r = g = b = 0; no sky:
 * sky_enabled must be 0), as rt_set_shading does for a handle; NULL turns it
 * off.  The server's record_mask must hold status, phi, r_hit, g and the
 * pixels, else RT_ERR_INVALID_ARG. */
rt_status rt_server_set_shading(rt_server* s, const rt_shading* shading);

/* Allocation-free bundle trace.  No counterpart in the reference: its compute
 * executor always owns its device buffers and grows them on demand.
 * Mixed-precision tables run the single-kernel form (mixed_single_kernel = 1):
 * the two-pass form needs buffers for parked rays.
 *
 * For callers that cannot allocate device memory at dispatch time: a host
 * that has reserved the whole device for its own pool allocator (a serving
 * process or an ML framework's caching allocator, where an outside cudaMalloc
 * fails or fragments the pool), a frame loop for which the implicit device
 * synchronisation of cudaFree is too costly, or a plugin with no
 * initialise/shutdown hooks to own an rt_handle.  The call needs no handle and
 * calls no cudaMalloc, cudaFree or other allocating routine.
 *
 * Scratch: one static device array per device, RT_NOALLOC_SCRATCH_BYTES
 * (15,104) bytes: the ray-queue counter and the launch counters (256 bytes,
 * zeroed on `stream` by every call before its launch) and a table of at most
 * RT_NOALLOC_MAX_BUNDLES bundle descriptors (written by every call).  A longer
 * table is rejected with RT_ERR_INVALID_ARG.  The outputs need no clearing:
 * every ray of the table is written.
 *
 * The first call on a device does its set-up (scratch address lookup, kernel
 * loading).  The call cannot be captured into a CUDA graph: it uploads the
 * bundle table from its own stack frame, which a replay could not read again,
 * so on a stream that is capturing it returns RT_ERR_INVALID_ARG before
 * enqueuing anything (the capture stays valid).  The caller's current device
 * is restored before the call returns.
 * Calls that overlap in time on one device share the one scratch array and
 * race: serialise them (one stream, or events between streams).
 *
 * cams / n_bundles / offsets / pixels / rays / capacity: as
 * rt_trace_bundles_device (device output pointers).  cfg: launch shape, NULL
 * for the defaults.  stream: a cudaStream_t, NULL = the legacy default stream;
 * the work is enqueued and not waited for (the bundle table is read from
 * host memory before the call returns).  error (optional): receives a
 * NUL-terminated message of at most error_len bytes on failure. */
#define RT_NOALLOC_MAX_BUNDLES 32
#define RT_NOALLOC_SCRATCH_BYTES 15104
rt_status rt_trace_bundles_noalloc(int device_ordinal, const rt_camera* cams, uint32_t n_bundles,
                                   const uint64_t* offsets, rt_pixel_out* pixels, const rt_ray_out* rays,
                                   size_t capacity, const rt_launch_config* cfg, void* stream, char* error,
                                   size_t error_len);

#ifdef __cplusplus
}
#endif

#endif
