// rt_shade.cu -- pixel shading pass (GpuPixelOutput's colour) for sm_100a.
//
// After a trace, one thread per ray turns the ray's radiance into the pixel's
// sRGB colour, as the reference's CPU image path does
// (software_compute_engine.hpp:1538-1611, 1734-1808, 3150-3252).  With the
// translucent-disk continuation (the handle's dispatches) the tracers record
// every disk crossing of a ray and this pass shades them in order at the
// throughput left, each with the descriptor of the source whose disk it
// crossed (multi-source scenes: one per source); without it (the server) the
// record's first hit (class, r_hit, phi, g) is shaded here as the thin disk at
// the crossing (AccretionDiskModel::shade,
// render/accretion_disk/accretion_disk_model.hpp:245-316, with the
// Novikov-Thorne base temperature of hydro model 1,
// render/accretion_disk/hydro_disk_shading.hpp:160-171).  The radiance is
// tonemapped (apply_tonemapping, :3461-3516).  Hydro model 2 replaces the
// crossings by the light the tracer gathered in the Fishbone-Moncrief torus.
// With the sky on, a ray that escapes, or ends outside 3 r_s with throughput
// left, adds the procedural sky (rt_sky.cuh) at its exit direction: recorded
// by the Boyer-Lindquist and multi-source tracers, and formed here from the
// tail record of a Kerr-Schild ray's end.  The sky's layers run between block
// barriers (one 16-warp block per SM), so that an SM's warps share one phase's
// code in the instruction cache.
//
// Per-camera constants (the resolved profile, the Novikov-Thorne flux
// normalisation, the spectral table of the blackbody colour) are computed on
// the host; the same helpers run on both sides.  Float is used where the
// reference uses float (the pattern and noise), double elsewhere.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "rt_device.cuh"
#include "rt_internal.h"
#include "rt_shade.cuh"
#include "rt_sky.cuh"

namespace relsim {

namespace {

// CIE 1931 colour-matching functions, multi-lobe Gaussian fit (Wyman, Sloan &
// Shirley, JCGT 2013), as optics/cie_observer.hpp:24-45 uses them.
double lobe(double x, double alpha, double mu, double s1, double s2) {
    const double s = (x < mu) ? s1 : s2;
    const double t = (x - mu) / s;
    return alpha * std::exp(-0.5 * t * t);
}

double temperature_shape(double u, double exponent, double zero_torque) {
    const double boundary = mxd(1.0 - zero_torque * std::sqrt(u), 0.0);
    return std::pow(u, exponent) * std::pow(boundary, 0.25);
}

__device__ __forceinline__ float to_srgb(double v) {
    if (v <= 0.0031308) return static_cast<float>(12.92 * v);
    return static_cast<float>(1.055 * pow(v, 1.0 / 2.4) - 0.055);
}

__device__ __forceinline__ double aces(double x) {
    return cd((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0, 1.0);
}


// Sky-lookup direction at the end of a Kerr-Schild ray from its tail record
// (TailField): the end interpolated to the threshold radius on the last step's
// Hermite interpolant when a threshold is set, then -dx/dlambda of that state,
// normalised (software_compute_engine.hpp:1771-1775).
__device__ __noinline__ void ks_tail_direction(const double* __restrict__ rec, double* e) {
    double y[6];
    const double target = rec[TL_TARGET], M = rec[TL_M], a = rec[TL_A];
    if (target > 0.0) {
        hermite(rec + TL_Y0, rec + TL_F0, rec + TL_Y1, rec + TL_F1, rec[TL_H],
                crossing_fraction(rec + TL_Y0, rec + TL_F0, rec + TL_Y1, rec + TL_F1, rec[TL_H], a, target), 6, y);
    } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) y[k] = rec[TL_Y1 + k];
    }
    double k[3], hf;
    ks_field64(y, M, a, k, hf);
    const double sv = 1.0 + k[0] * y[3] + k[1] * y[4] + k[2] * y[5];
    const double v[3] = {y[3] - 2.0 * hf * sv * k[0], y[4] - 2.0 * hf * sv * k[1], y[5] - 2.0 * hf * sv * k[2]};
    const double inv = 1.0 / fmax(sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), 1e-12);
#pragma unroll
    for (int c = 0; c < 3; ++c) e[c] = -v[c] * inv;
}

__global__ void __launch_bounds__(512) shade_kernel(const ShadeDesc* __restrict__ Dp,
                                                    const uint32_t* __restrict__ status,
                                                    const double* __restrict__ r_hit,
                                                    const double* __restrict__ phi,
                                                    const double* __restrict__ g, ContOut cont,
                                                    rt_pixel_out* __restrict__ pixels, uint64_t n) {
    const ShadeDesc& D = *Dp;  // the camera's hole (and the tonemap)
    // block-uniform iterations: the sky's layers run between block barriers
    const bool sky_pass = D.sky_on && cont.cross && (cont.exit || cont.tail);
    for (uint64_t base = blockIdx.x * static_cast<uint64_t>(blockDim.x); base < n;
         base += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        const bool live = i < n;
        double acc[3] = {0.0, 0.0, 0.0};
        double e[3] = {0.0, 0.0, 0.0}, thr = 1.0;
        bool sky_here = false;
        if (!live) {
        } else if (cont.cross) {
            // translucent disk (software_compute_engine.hpp:1660, 1743-1796): the
            // crossings in order, each at the throughput left, while more than 0.01
            // is left; the pixel's redshift is the last crossing's and its flags add
            // the way the ray ended, if the throughput lasted to the end
            const uint32_t info = cont.info[i];
            const uint32_t n_cross = info & CI_COUNT_MASK;
            const uint32_t bodies = cont.body ? cont.body[i] : 0u;  // source of each crossing
            double last_g = 1.0;
            if (cont.vol) {
                // hydro model 2: the light the tracer gathered in the torus
                // (no thin-disk crossings); its redshift is the last segment's
                const double* V = cont.vol + i * VL_COUNT;
                if (V[VL_HIT] != 0.0) {
                    acc[0] = V[VL_R];
                    acc[1] = V[VL_G];
                    acc[2] = V[VL_B];
                    thr = V[VL_THR];
                    pixels[i].status_flags |= RT_PIXEL_ACCRETION_DISK_HIT;
                    pixels[i].redshift = static_cast<float>(V[VL_Z]);
                }
            }
            for (uint32_t k = 0; k < n_cross && thr > kMinThroughput; ++k) {
                double sh[4];
                const double gk = cont.cross[(3 * k + 2) * cont.stride + i];
                disk_radiance(Dp[(bodies >> (4u * k)) & 15u], cont.cross[(3 * k) * cont.stride + i],
                              cont.cross[(3 * k + 1) * cont.stride + i], gk, sh);
                acc[0] += thr * sh[0];
                acc[1] += thr * sh[1];
                acc[2] += thr * sh[2];
                thr *= 1.0 - sh[3];
                last_g = gk;
            }
            // how the ray ended (software_compute_engine.hpp:1766-1795): with throughput
            // left, a capture absorbs it; an escape, or an end outside 3 r_s, sees the sky
            const uint32_t fate = (info >> CI_FATE_SHIFT) & 15u;
            uint32_t add = 0;
            if (thr > kMinThroughput) {
                if (fate == RT_RAY_CAPTURED) add = RT_PIXEL_HORIZON_ABSORBED;
                else if (fate == RT_RAY_ESCAPED || !(info & CI_INSIDE_3RS)) add = RT_PIXEL_CELESTIAL_HIT;
            }
            pixels[i].status_flags |= add;
            if (n_cross > 0) pixels[i].redshift = static_cast<float>(last_g);
            if (sky_pass && add == RT_PIXEL_CELESTIAL_HIT) {
                sky_here = true;
                if (cont.tail) {
                    ks_tail_direction(cont.tail + i * TL_COUNT, e);
                } else {
                    e[0] = cont.exit[i];
                    e[1] = cont.exit[cont.stride + i];
                    e[2] = cont.exit[2 * cont.stride + i];
                }
            }
        } else if (status[i] == RT_RAY_DISK) {
            double sh[4];
            disk_radiance(D, r_hit[i], phi[i], g[i], sh);
            acc[0] = sh[0];
            acc[1] = sh[1];
            acc[2] = sh[2];
        }
        // the sky behind the rays that see it, at the throughput left; every
        // thread of the block takes the layers' barriers
        if (sky_pass && __syncthreads_or(sky_here)) {
            float sky_rgb[3];
            // barriers after the nebulae (the noise code) and after the stars: the
            // sparse layers between run as one phase (measured 9.4 ms for the
            // 2048^2 image, against 9.7 with a barrier after every layer and 11.1
            // with none)
            sky::sample_phased(D.sky, e[0], e[1], e[2], D.fov, D.time, sky_here, sky_rgb, [](int layer) {
                if (layer == sky::L_NEBULAE || layer == sky::L_STARS) __syncthreads();
            });
            if (sky_here) {
                acc[0] += thr * static_cast<double>(sky_rgb[0]);
                acc[1] += thr * static_cast<double>(sky_rgb[1]);
                acc[2] += thr * static_cast<double>(sky_rgb[2]);
            }
        }
        if (!live) continue;
        // apply_tonemapping (software_compute_engine.hpp:3461-3516)
        const double k = exp2(D.exposure);
        double r = mxd(0.0, acc[0] * k), gg = mxd(0.0, acc[1] * k), b = mxd(0.0, acc[2] * k);
        if (D.tonemap == 1u) {
            r = aces(r);
            gg = aces(gg);
            b = aces(b);
        } else if (D.tonemap == 2u) {
            const double lum = 0.2126 * r + 0.7152 * gg + 0.0722 * b;
            if (lum > 0.0) {
                const double mapped = log10(1.0 + lum * 100.0) / log10(1.0 + 10000.0);
                const double s = cd(mapped / lum, 0.0, 1.0);
                r = cd(r * s, 0.0, 1.0);
                gg = cd(gg * s, 0.0, 1.0);
                b = cd(b * s, 0.0, 1.0);
            }
        } else if (D.tonemap == 3u) {
            r = (r * (1.0 + r / 25.0)) / (1.0 + r);
            gg = (gg * (1.0 + gg / 25.0)) / (1.0 + gg);
            b = (b * (1.0 + b / 25.0)) / (1.0 + b);
        } else {
            r = cd(r, 0.0, 1.0);
            gg = cd(gg, 0.0, 1.0);
            b = cd(b, 0.0, 1.0);
        }
        reinterpret_cast<float4*>(pixels + i)[0] = make_float4(to_srgb(r), to_srgb(gg), to_srgb(b), 1.0f);
    }
}

double temperature_shape_peak(double exponent, double zero_torque) {
    double lo = 1e-4, hi = 1.0;
    for (int it = 0; it < 48; ++it) {  // ternary search on a unimodal shape
        const double a = lo + (hi - lo) / 3.0;
        const double b = hi - (hi - lo) / 3.0;
        if (temperature_shape(a, exponent, zero_torque) < temperature_shape(b, exponent, zero_torque)) lo = a;
        else hi = b;
    }
    return mxd(temperature_shape(0.5 * (lo + hi), exponent, zero_torque), temperature_shape(1.0, exponent, zero_torque));
}

}  // namespace

bool build_shade_desc(const rt_camera& cam, const rt_shading& s, ShadeDesc& d) {
    if (s.hydro_model > 2u || s.sky_enabled > 1u || s.tonemapping_mode > 3u) return false;
    d = ShadeDesc{};
    // spectral table (accretion_disk_model.hpp:52-69)
    const double step = (780.0 - 380.0) / 32.0;
    for (int i = 0; i <= 32; ++i) {
        const double lnm = 380.0 + static_cast<double>(i) * step;
        const double trap = (i == 0 || i == 32) ? 0.5 : 1.0;
        d.lambda_um[i] = lnm * 1e-3;
        d.weight[i][0] = trap * (lobe(lnm, 1.056, 599.8, 37.9, 31.0) + lobe(lnm, 0.362, 442.0, 16.0, 26.7) -
                                 lobe(lnm, 0.065, 501.1, 20.4, 26.2));
        d.weight[i][1] = trap * (lobe(lnm, 0.821, 568.8, 46.9, 40.5) + lobe(lnm, 0.286, 530.9, 16.3, 31.1));
        d.weight[i][2] = trap * (lobe(lnm, 1.217, 437.0, 11.8, 36.0) + lobe(lnm, 0.681, 459.0, 26.0, 13.8));
    }
    // resolve_primary_profile + finalize (accretion_disk_model.hpp:180-196)
    static_assert(sizeof(rt_disk_profile) == 32 * sizeof(float), "GpuDiskProfile layout");
    std::copy_n(reinterpret_cast<const float*>(&s.disk), 32, d.profile);
    float* P = d.profile;
    P[DP_PEAK_T] = static_cast<float>(s.disk_temperature_scale_k);
    P[DP_FLOOR_T] = static_cast<float>(s.disk_temperature_floor_k);
    P[DP_SATURATION] = static_cast<float>(s.disk_color_saturation);
    P[DP_BEAMING] = static_cast<float>(s.disk_doppler_beaming_exponent);
    P[DP_PEAK_T] = cf(P[DP_PEAK_T], 1000.0f, 200000.0f);
    P[DP_FLOOR_T] = cf(P[DP_FLOOR_T], 0.0f, P[DP_PEAK_T]);
    const double peak = temperature_shape_peak(static_cast<double>(P[DP_T_EXPONENT]), static_cast<double>(P[DP_ZERO_TORQUE]));
    P[DP_T_NORMALIZATION] = static_cast<float>(1.0 / mxd(peak, 1e-6));
    double xyz[3];
    planck_xyz(d.lambda_um, d.weight, static_cast<double>(P[DP_PEAK_T]), xyz);
    P[DP_REF_LUMINANCE] = static_cast<float>(mxd(xyz[1], 1e-30));

    // disk geometry and the camera's detail factor (software_compute_engine.hpp:3800-3836)
    const double m = mxd(cam.metric_mass, 1e-4);
    const double a = cd(cam.metric_spin, -0.999 * m, 0.999 * m);
    const double inner = (cam.disk_inner_radius > 0.0) ? cam.disk_inner_radius : kerr_isco_radius(m, a);
    d.mass = mxd(m, 1e-9);
    d.disk_spin = a;
    d.inner = mxd(inner, 1e-9);
    d.outer = mxd(cam.disk_outer_radius, d.inner * 1.0001);
    d.time = s.time;
    d.exposure = s.camera_exposure;
    d.tonemap = s.tonemapping_mode;
    d.hydro_model = s.hydro_model;
    const double rh = (std::fabs(a) > 1e-12) ? (m + std::sqrt(mxd(m * m - a * a, 0.0))) : 2.0 * m;
    const double r_obs = mxd(cam.observer_position[1], rh * 1.02);
    const double pixel = cam.field_of_view_rad / mxd(static_cast<double>(cam.screen_width), 1.0);
    d.detail = cd((2.0 * rh / r_obs) / mxd(pixel * 24.0, 1e-9), 0.0, 1.0);
    d.pattern_omega = orbital_omega(d.mass, a, std::sqrt(d.inner * d.outer));
    // the procedural sky (GpuSkyProfile image) and the camera's field of view
    static_assert(sizeof(rt_sky_profile) == sizeof(SkyProfile), "sky profile layout");
    std::memcpy(&d.sky, &s.sky, sizeof d.sky);
    d.sky_on = (s.sky_enabled == 1u && d.sky.enabled != 0u) ? 1u : 0u;
    d.fov = cam.field_of_view_rad;

    // Novikov-Thorne disk of (M, a): ISCO, Page-Thorne roots, peak flux over
    // 192 log-spaced radii (hydro_disk_shading.hpp:44-62)
    d.nt_m = d.mass;
    d.nt_a_star = cd(a / d.mass, -0.999999999, 0.999999999);
    {
        const double as = d.nt_a_star;
        const double z1 = 1.0 + std::cbrt(1.0 - as * as) * (std::cbrt(1.0 + as) + std::cbrt(1.0 - as));
        const double z2 = std::sqrt(3.0 * as * as + z1 * z1);
        const double root = std::sqrt(mxd(0.0, (3.0 - z1) * (3.0 + z1 + 2.0 * z2)));
        d.nt_r_isco = d.mass * ((as >= 0.0) ? (3.0 + z2 - root) : (3.0 + z2 + root));
        d.nt_x0 = std::sqrt(d.nt_r_isco / d.mass);
        const double psi = std::acos(cd(as, -1.0, 1.0)) / 3.0;
        d.nt_x1 = 2.0 * std::cos(psi - kPiD / 3.0);
        d.nt_x2 = 2.0 * std::cos(psi + kPiD / 3.0);
        d.nt_x3 = -2.0 * std::cos(psi);
    }
    {
        const double lo = mxd(d.inner, d.nt_r_isco * 1.0001);
        const double hi = mxd(d.outer, lo * 1.01);
        const double ratio = hi / lo;
        double pk = 0.0;
        for (int i = 0; i < 192; ++i) pk = mxd(pk, nt_flux(d, lo * std::pow(ratio, static_cast<double>(i) / 191.0)));
        d.nt_flux_peak = (pk > 1e-300) ? pk : 1.0;
        d.nt_rate_factor = std::pow(mxd(static_cast<double>(s.accretion_rate_scale), 1e-6), 0.25);
    }
    // hydro model 2: the Fishbone-Moncrief torus of the camera's hole
    // (HydroDiskContext::build_torus, hydro_disk_shading.hpp:76-110)
    if (s.hydro_model == 2u) {
        const torus::TorusContext c = torus::make_torus(d.mass, a, static_cast<double>(s.torus_inner_radius),
                                                        static_cast<double>(s.torus_center_radius));
        d.fm_valid = c.valid ? 1u : 0u;
        d.fm_m = c.t.m;
        d.fm_a = c.t.a;
        d.fm_rh = c.t.rh;
        d.fm_l = c.t.l;
        d.fm_w_in = c.t.w_in;
        d.fm_h_max = c.h_max;
        d.fm_inner = c.inner_bound;
        d.fm_outer = c.outer_bound;
        d.fm_exponent = 1.0 / mxd(static_cast<double>(s.adiabatic_index) - 1.0, 1e-3);
        d.fm_kappa = static_cast<double>(s.optical_depth_scale) * mxd(static_cast<double>(P[DP_OPACITY_SCALE]), 0.0);
        d.fm_density = mxd(static_cast<double>(s.sampling_density), 0.1);
    }
    return true;
}

// A multi-source body's descriptor from the scene's base descriptor: its disk
// profile as it stands (GpuBodyData::disk), its geometry; the thin procedural
// model at detail 1, as trace_multi_source shades every source
// (software_compute_engine.hpp:3172-3185).
void build_source_shade_desc(const ShadeDesc& base, const float* profile, double mass, double spin, double inner,
                             double outer, ShadeDesc& d) {
    d = base;
    if (profile) std::copy_n(profile, 32, d.profile);
    d.mass = mxd(mass, 1e-9);
    d.disk_spin = spin;
    d.inner = mxd(inner, 1e-9);
    d.outer = mxd(outer, d.inner * 1.0001);
    d.detail = 1.0;
    d.hydro_model = 0u;
    d.pattern_omega = orbital_omega(d.mass, spin, std::sqrt(d.inner * d.outer));
}

void launch_shade(const ShadeDesc* desc, const uint32_t* status, const double* r_hit, const double* phi,
                  const double* g, ContOut cont, rt_pixel_out* pixels, uint64_t n, void* stream) {
    if (n == 0) return;
    // 512 threads: one block of 16 warps per SM at 128 registers, so that the
    // warps of an SM run the same sky layer
    const uint64_t blocks = std::min<uint64_t>((n + 511) / 512, 148ull * 8);
    shade_kernel<<<static_cast<unsigned>(blocks), 512, 0, static_cast<cudaStream_t>(stream)>>>(desc, status, r_hit,
                                                                                                phi, g, cont, pixels, n);
}

}  // namespace relsim
