/*
 * ks_oracle.h -- FP64 CPU oracle for the backward null-geodesic tracer.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * engine's Kerr-Schild null-ray path, used as the checker for the CUDA
 * kernels.  Only tests/, the smoke check in __graft_entry__.py and the
 * cpu_baseline leg of bench.py may load it.  No product code path calls it.
 *
 * What it restates (reference = Wartets/Relativity-Simulator):
 *   - Kerr-Schild field and Hamiltonian RHS with p_t = -1
 *       include/relativistic/core/kerr_schild_null_integrator.hpp:31-44, 72-114
 *   - BL <-> KS position maps with phi unwrapping  (:47-69)
 *   - static-observer tetrad and initial null momentum  (:142-194)
 *   - pinhole camera + tetrad ray generation
 *       include/relativistic/observer/camera_projections.hpp:27-40
 *       include/relativistic/render/software_compute_engine.hpp:3838-3938
 *   - Dormand-Prince 5(4) tableau, max-norm error, accept/reject scaling
 *       include/relativistic/integrators/rk45_adaptive.hpp:196-311
 *   - PI30 step controller  include/relativistic/integrators/step_controller.hpp:44-78
 *   - constraint projection, closest-root quadratic  rk45_adaptive.hpp:91-139
 *   - ISCO  software_compute_engine.hpp:1052-1061
 *   - disk redshift  include/relativistic/render/accretion_disk/accretion_disk_model.hpp:205-225
 *   - Carter constant  include/relativistic/metrics/kerr_invariants.hpp:21-58
 *   - radial quartic of the Carter classifier
 *       include/relativistic/optics/carter_ray_classifier.hpp:116-140
 */
#ifndef RELSIM_KS_ORACLE_H
#define RELSIM_KS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Ray classes (same numbering as the CUDA library's RT_RAY_* codes). */
enum {
    ORC_RAY_UNFINISHED = 0, /* step budget exhausted */
    ORC_RAY_CAPTURED = 1,   /* r_BL < capture_scale * r_+ (or non-finite state) */
    ORC_RAY_ESCAPED = 2,    /* r_BL > escape_radius */
    ORC_RAY_DISK = 3        /* first z = 0 crossing with r in [r_in, r_out] */
};
enum {
    ORC_FLAG_NONFINITE = 1u << 0,
    ORC_FLAG_STEP_UNDERFLOW = 1u << 1,
    ORC_FLAG_MAX_STEPS = 1u << 2,
    ORC_FLAG_EARLY_CAPTURE = 1u << 3,
    ORC_FLAG_DIVERGED = 1u << 4 /* multi-source: |p| above ORC_MS_MAX_MOMENTUM */
};

/* A ray is declared captured before reaching capture_scale * r_+ when it is
 * inside the disk's inner edge, moving inwards, and its radial potential has
 * no turning point outside r_+ by at least this margin (signed distance to the
 * critical curve, in M). */
#define ORC_EARLY_CAPTURE_MARGIN 1e-4

typedef struct orc_camera {
    double observer_position[4]; /* t, r, theta, phi (Boyer-Lindquist) */
    double tetrad_e1[4];         /* forward  (spatial part in [1..3]) */
    double tetrad_e2[4];         /* right */
    double tetrad_e3[4];         /* up */
    double field_of_view_rad;
    double metric_mass;
    double metric_spin;
    double escape_radius;
    double capture_scale;        /* captured when r_BL < capture_scale * r_+ */
    double disk_inner_radius;    /* <= 0 selects r_ISCO(a) */
    double disk_outer_radius;    /* <= 0 disables the disk */
    double rtol;
    double atol;
    double step_cap_fraction;    /* |h| <= c * max(r_BL - r_+, 0.01 M) */
    double initial_step_fraction;/* |h0| = f * r_obs */
    double projection_tol;       /* project when |H| > tol * (1 + |p|^2) */
    uint32_t screen_width;
    uint32_t screen_height;
    uint32_t max_steps;          /* step attempts, accepted + rejected */
    uint32_t early_capture;      /* 1: stop once capture is certain (Carter test) */
} orc_camera;

typedef struct orc_ray {
    uint32_t status;
    uint32_t flags;
    uint32_t steps_accepted;
    uint32_t steps_rejected;
    double r, theta, phi;        /* final BL position */
    double r_hit;                /* disk-hit radius, NaN when no hit */
    double g;                    /* disk redshift factor, 1 when no hit */
    double lambda;               /* affine parameter at termination */
    double dH;                   /* max |H| before projection */
    double dE;                   /* E recomputed from the null condition - 1 */
    double dLz;                  /* L_z(end) - L_z(start) */
    double dQ;                   /* Q(end) - Q(start) */
    double db_shadow;            /* signed distance to the critical curve (M) */
    double exit_dir[3];          /* escaped rays: the sky-lookup direction at the terminal state
                                    (Kerr-Schild: -dx/dlambda normalised, software_compute_engine.hpp:
                                    1771-1775; multi-source: the superposed flow, :3220-3224;
                                    Boyer-Lindquist: the local-frame velocity as a direction of
                                    travel, :1581-1589); NaN otherwise */
    uint32_t body;               /* the body the ray ended on: the source of its first disk hit or of
                                    its capture (0: the camera's hole); ORC_BODY_NONE otherwise */
    uint32_t pad;
} orc_ray;
#define ORC_BODY_NONE 0xFFFFFFFFu

/* Translucent-disk continuation of a ray (software_compute_engine.hpp:1734-1765,
 * :1771-1795): the reference's image path does not end a ray at the disk; each
 * crossing adds the disk's radiance at the remaining throughput and the ray
 * goes on to its capture or escape, where the sky behind adds in. */
#define ORC_MAX_CROSSINGS 8
typedef struct orc_cont {
    uint32_t n_cross;            /* disk crossings recorded, in order along the backward ray */
    uint32_t fate;               /* class at the ray's end (ORC_RAY_*) */
    double cross_r[ORC_MAX_CROSSINGS];
    double cross_phi[ORC_MAX_CROSSINGS];
    double cross_g[ORC_MAX_CROSSINGS];
    double exit_dir[3];          /* escaped at its end: the sky-lookup direction; NaN otherwise */
    uint32_t cross_src[ORC_MAX_CROSSINGS]; /* multi-source: the source whose disk crossing k is on (else 0) */
    uint32_t near_source;        /* multi-source: the end point lies within 6 m of a source */
    uint32_t pad;
} orc_cont;

/* Hydro model 2, the Fishbone-Moncrief torus: its constants with the resolved
 * disk profile (shade_oracle.c orc_fm_context), one chord's emission and
 * absorption (orc_fm_segment: radiance r, g, b, opacity, redshift) and the
 * accumulation into a ray's gathered light (orc_fm_accumulate: r, g, b,
 * throughput, redshift, seen; all 0 before the first emitting segment). */
typedef struct orc_fm {
    double m, a, rh, l, w_in, h_max, inner, outer, exponent, kappa, density;
    uint32_t valid, closed;
    float profile[32];
} orc_fm;
void orc_fm_context(double mass, double spin, double r_in_units, double r_center_units, double gamma,
                    double optical_depth_scale, double sampling_density, const float resolved_profile[32], orc_fm* out);
void orc_fm_segment(const orc_fm* t, const double from[3], const double to[3], double l_over_e, double out[5]);
void orc_fm_accumulate(const orc_fm* t, const double from[3], const double to[3], double l_over_e, double vol[6]);
/* Trace with the torus: every accepted step's chord between the Boyer-Lindquist
 * points of its ends, as Cartesian, is accumulated into vol[6 * i] (the camera
 * as given; the caller turns the thin disk and early capture off, as the
 * library does for hydro model 2). */
void orc_trace_volume(const orc_camera* cam, const orc_fm* fm, const uint64_t* pixel_index, uint64_t first,
                      uint64_t count, orc_ray* out, orc_cont* cont, double* vol, int threads);
/* The same for the Boyer-Lindquist Kerr-Newman trace (chords between the
 * steps' Boyer-Lindquist points; L / E as u^phi r^2 sin^2 theta at each step's
 * end, as the reference's metric-type path takes it). */
void orc_bl_trace_volume(const orc_camera* cam, double charge, const orc_fm* fm, const uint64_t* pixel_index,
                         uint64_t first, uint64_t count, orc_ray* out, orc_cont* cont, double* vol, int threads);

/* --- single-function checks (pinned against the reference) --- */
void orc_ks_field(const double x[3], double mass, double spin, double* r, double* h, double k[3]);
void orc_ks_rhs(const double y[6], double mass, double spin, double dy[6]);
void orc_ks_position_from_bl(double r, double theta, double phi, double spin, double out[3]);
void orc_bl_from_ks(const double x[3], double spin, double previous_phi, double out[3]);
void orc_initial_momentum(const double x[3], double mass, double spin, const double outward[3], double p[3]);
double orc_isco_radius(double mass, double spin);
double orc_redshift_at(double mass, double spin, double radius, double lz);
void orc_pinhole_ray(double u, double v, double fov, double n[3]);
double orc_pi30_factor(double err, double err_prev, int has_history, double order_p1);
double orc_hamiltonian(const double y[6], double mass, double spin);
double orc_carter_q(const double y[6], double mass, double spin);
double orc_shadow_distance(double mass, double spin, double lz, double q);

/* Initial state of pixel (px, py): y0 = (x, p), returns L_z. */
double orc_ray_initial_state(const orc_camera* cam, uint32_t px, uint32_t py, double y0[6]);

/* One DP45 attempt from y with step h (no control): y_new and the error norm. */
double orc_dp45_attempt(const orc_camera* cam, const double y[6], double h, double y_new[6]);

/* Trace pixels.  pixel_index == NULL traces the contiguous range
 * [first, first + count) of row-major pixel indices, else the listed ones.
 * threads <= 0 uses all online cores. */
void orc_trace(const orc_camera* cam, const uint64_t* pixel_index, uint64_t first, uint64_t count,
               orc_ray* out, int threads);
/* The same with the translucent-disk continuation: `out` describes each ray's
 * first hit as orc_trace does, `cont` its crossings and end. */
void orc_trace_cont(const orc_camera* cam, const uint64_t* pixel_index, uint64_t first, uint64_t count,
                    orc_ray* out, orc_cont* cont, int threads);

/* --- multi-source Kerr-Schild superposition (ms_oracle.c) --- */
#define ORC_MS_MAX_SOURCES 16
/* A multi-source ray whose momentum exceeds this (E = 1 units) is inside a
 * horizon-like region of the superposed field, where the sum of the sources'
 * fields traps it without reaching any single source's horizon: it is
 * captured, with ORC_FLAG_DIVERGED. */
#define ORC_MS_MAX_MOMENTUM 1e3

/* A black-hole body beside the camera's own hole (GpuBodyData with preset 8). */
typedef struct orc_source {
    double position[3];
    double mass;
    double spin_parameter;   /* a / m, clamped to [-0.9999, 0.9999] */
    double axis[3];          /* spin axis (normalised; zero selects +z) */
    double disk_enabled;     /* > 0.5: thin disk */
    double disk_inner_scale; /* inner radius = max(scale, 1) * r_ISCO */
    double disk_outer_units; /* outer radius = max(units * m, 1.05 * inner) */
} orc_source;

/* Source table with local frames; source 0 is the camera's hole at the origin. */
typedef struct orc_ms_table {
    uint32_t count;
    double pos[ORC_MS_MAX_SOURCES][3];
    double mass[ORC_MS_MAX_SOURCES];
    double axis[ORC_MS_MAX_SOURCES][3];
    double spin[ORC_MS_MAX_SOURCES];
    double fx[ORC_MS_MAX_SOURCES][3];
    double rh[ORC_MS_MAX_SOURCES];
    double fy[ORC_MS_MAX_SOURCES][3];
    double req[ORC_MS_MAX_SOURCES];
    double disk_in[ORC_MS_MAX_SOURCES];  /* < 0: no disk */
    double disk_out[ORC_MS_MAX_SOURCES];
} orc_ms_table;

void orc_ms_build(const orc_camera* cam, const orc_source* src, uint32_t n, orc_ms_table* t);
void orc_ms_rhs(const orc_ms_table* t, const double y[6], double dy[6]);
double orc_ms_hamiltonian(const orc_ms_table* t, const double y[6]);
void orc_ms_initial_momentum(const orc_ms_table* t, const double x[3], const double outward[3], double p[3]);
int orc_ms_inside_horizon(const orc_ms_table* t, const double x[3]);
void orc_ms_initial_state(const orc_camera* cam, const orc_ms_table* t, uint32_t px, uint32_t py, double y0[6]);
/* The same with the translucent-disk continuation (trace_multi_source,
 * software_compute_engine.hpp:3150-3216): every crossing of a step in order
 * along the ray, each on the disk of cross_src[k]; `out` describes the first
 * hit, `cont` the crossings and the end. */
void orc_ms_trace_cont(const orc_camera* cam, const orc_ms_table* t, const uint64_t* pixel_index, uint64_t first,
                       uint64_t count, orc_ray* out, orc_cont* cont, int threads);
void orc_ms_trace(const orc_camera* cam, const orc_ms_table* t, const uint64_t* pixel_index, uint64_t first,
                  uint64_t count, orc_ray* out, int threads);

/* --- Boyer-Lindquist Kerr-Newman form (bl_oracle.c) ---
 * State y = (r, theta, phi, u^t, u^r, u^theta, u^phi), u future-directed and
 * traced with steps h < 0.  Metric components in the order
 * (g_tt, g_tphi, g_rr, g_thth, g_phiphi).  In orc_ray: dE = E / E0 - 1,
 * dLz = (L - L0) / E0, dQ = (Q - Q0) / E0^2, db_shadow from the Kerr-Newman
 * radial potential. */
double orc_kn_horizon(double mass, double spin, double charge);
void orc_kn_metric(double mass, double spin, double charge, double r, double theta, double g[5]);
void orc_kn_metric_derivs(double mass, double spin, double charge, double r, double theta, double dr[5],
                          double dth[5]);
void orc_bl_rhs(double mass, double spin, double charge, const double y[7], double dy[7]);
double orc_bl_null_residual(double mass, double spin, double charge, const double y[7]);
void orc_bl_invariants(double mass, double spin, double charge, const double y[7], double out[3]);
double orc_kn_shadow_distance(double mass, double spin, double charge, double xi, double eta);
void orc_bl_zamo_ray(double mass, double spin, double charge, double r, double theta, double n_r, double n_th,
                     double n_ph, double u[4]);
void orc_bl_initial_state(const orc_camera* cam, double charge, uint32_t px, uint32_t py, double y0[7]);
void orc_bl_trace(const orc_camera* cam, double charge, const uint64_t* pixel_index, uint64_t first, uint64_t count,
                  orc_ray* out, int threads);
/* The same with the translucent-disk continuation (as orc_trace_cont). */
void orc_bl_trace_cont(const orc_camera* cam, double charge, const uint64_t* pixel_index, uint64_t first,
                       uint64_t count, orc_ray* out, orc_cont* cont, int threads);

/* --- pixel shading tail (shade_oracle.c) ---
 * Disk profiles are GpuDiskProfile's 32 floats in declaration order.  A
 * surface point is (mass, spin, inner, outer, radius, azimuth, redshift, time,
 * detail); shading output is (r, g, b, opacity). */
void orc_planck_xyz(double temperature_k, double xyz[3]);
void orc_blackbody_rgb(double temperature_k, double reference_luminance, double rgb[3]);
void orc_resolve_profile(const float in[32], const double overrides[4], float out[32]);
void orc_nt_context(double mass, double spin, double inner, double outer, float accretion_rate_scale, double out[2]);
void orc_disk_shade(const float profile[32], const double point[9], uint32_t hydro_model, float accretion_rate_scale,
                    double out[4]);
void orc_tonemap(const double rgb[3], uint32_t mode, double exposure_ev, float out[3]);
void orc_shade_pixel(const float resolved_profile[32], uint32_t hydro_model, float accretion_rate_scale,
                     uint32_t tonemap_mode, double exposure_ev, double mass, double disk_spin, double inner,
                     double outer, double time, double detail, uint32_t status, double r_hit, double phi, double g,
                     float out[3]);
void orc_shade_cont(const float resolved_profile[32], uint32_t hydro_model, float accretion_rate_scale,
                    uint32_t tonemap_mode, double exposure_ev, double mass, double disk_spin, double inner,
                    double outer, double time, double detail, uint32_t n_cross, const double* cross_r,
                    const double* cross_phi, const double* cross_g, float out[3]);

#ifdef __cplusplus
}
#endif

#endif
