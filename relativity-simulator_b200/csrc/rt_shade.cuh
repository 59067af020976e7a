// rt_shade.cuh -- disk shading on the device: the radiance and opacity of a
// thin-disk crossing (AccretionDiskModel::shade,
// render/accretion_disk/accretion_disk_model.hpp:245-316; the Novikov-Thorne
// base temperature of hydro model 1, hydro_disk_shading.hpp:160-171), used by
// the shading pass (rt_shade.cu); the continuation records the tracers write
// for it; and the Fishbone-Moncrief torus's chord integral of hydro model 2,
// which the tracers call step by step.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "rt_internal.h"
#include "rt_torus.cuh"

namespace relsim {

namespace {

constexpr double kPiD = 3.14159265358979323846;
constexpr double kTwoPiD = 2.0 * kPiD;

__host__ __device__ inline double cd(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }
__host__ __device__ inline double mxd(double a, double b) { return a < b ? b : a; }
__host__ __device__ inline float mxf(float a, float b) { return a < b ? b : a; }
__host__ __device__ inline float cf(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }

enum {
    DP_PEAK_T = 3, DP_FLOOR_T, DP_T_EXPONENT, DP_ZERO_TORQUE, DP_BEAMING, DP_BRIGHTNESS, DP_SATURATION,
    DP_TINT_STRENGTH, DP_OPACITY_SCALE, DP_TINT_R, DP_TINT_G, DP_TINT_B, DP_ROTATION, DP_RING_AMP, DP_RING_FREQ,
    DP_RING_SHARP, DP_ARMS, DP_PITCH, DP_SPIRAL_AMP, DP_TURB_AMP, DP_TURB_SCALE, DP_TURB_OCTAVES,
    DP_RADIAL_STRETCH, DP_GRAIN_AMP, DP_GRAIN_SCALE, DP_REF_LUMINANCE, DP_NOISE_SEED, DP_T_NORMALIZATION,
    DP_EDGE_SOFTNESS
};

// Planck radiance against the spectral table: XYZ (accretion_disk_model.hpp:71-88).
__host__ __device__ void planck_xyz(const double* lambda_um, const double (*w)[3], double temperature_k,
                                    double* xyz) {
    const double t = cd(temperature_k, 300.0, 400000.0);
    xyz[0] = xyz[1] = xyz[2] = 0.0;
    for (int i = 0; i <= 32; ++i) {
        const double lum = lambda_um[i];
        const double e = 14387.76877 / (lum * t);  // second radiation constant, um K
        if (e > 80.0) continue;
        const double l2 = lum * lum;
        const double rad = 1.0 / (l2 * l2 * lum * expm1(e));
        xyz[0] += rad * w[i][0];
        xyz[1] += rad * w[i][1];
        xyz[2] += rad * w[i][2];
    }
}

__device__ __forceinline__ double temperature_shape_d(double u, double exponent, double zero_torque) {
    const double boundary = mxd(1.0 - zero_torque * sqrt(u), 0.0);
    return pow(u, exponent) * pow(boundary, 0.25);
}

// Page & Thorne (1974) flux of the Novikov-Thorne disk (hydro/novikov_thorne.hpp:120-165, 295-325).
__host__ __device__ double nt_flux(const ShadeDesc& d, double r) {
    if (r < d.nt_r_isco) return 0.0;
    const double x = sqrt(r / d.nt_m);
    double f = 0.0;
    if (!(x < d.nt_x0)) {
        const double a = d.nt_a_star, x0 = d.nt_x0, x1 = d.nt_x1, x2 = d.nt_x2, x3 = d.nt_x3;
        f = x - x0;
        if (fabs(a) > 1e-15) f -= 1.5 * a * log(x / x0);
        f -= 3.0 * (x1 - a) * (x1 - a) / (x1 * (x1 - x2) * (x1 - x3)) * log(mxd((x - x1) / (x0 - x1), 1e-30));
        if (fabs(x2) > 1e-12)
            f -= 3.0 * (x2 - a) * (x2 - a) / (x2 * (x2 - x1) * (x2 - x3)) * log(mxd((x - x2) / (x0 - x2), 1e-30));
        f -= 3.0 * (x3 - a) * (x3 - a) / (x3 * (x3 - x1) * (x3 - x2)) * log(mxd((x - x3) / (x0 - x3), 1e-30));
        f = mxd(0.0, f);
    }
    const double x3 = x * x * x;
    const double den = x * (x3 + d.nt_a_star);
    if (den <= 1e-24) return 0.0;
    const double factor = (3.0 * d.nt_m * 1.0) / (8.0 * kPiD * (r * r * r));
    return mxd(0.0, factor * (f / den));
}

// lowbias32 integer hash (C. Wellons) and value noise on its lattice
// (accretion_disk_model.hpp:119-178).
__device__ __forceinline__ uint32_t lowbias32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ float lattice(int32_t x, int32_t y, int32_t z, uint32_t seed) {
    const uint32_t h = static_cast<uint32_t>(x) * 374761393U + static_cast<uint32_t>(y) * 668265263U +
                       static_cast<uint32_t>(z) * 2147483647U + seed * 1274126177U;
    return static_cast<float>(lowbias32(h) & 0x00FFFFFFU) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
}

__device__ float value_noise(float x, float y, float z, uint32_t seed) {
    const float fx0 = floorf(x), fy0 = floorf(y), fz0 = floorf(z);
    const int32_t xi = static_cast<int32_t>(fx0), yi = static_cast<int32_t>(fy0), zi = static_cast<int32_t>(fz0);
    const float fx = x - fx0, fy = y - fy0, fz = z - fz0;
    const float ux = fx * fx * (3.0f - 2.0f * fx);
    const float uy = fy * fy * (3.0f - 2.0f * fy);
    const float uz = fz * fz * (3.0f - 2.0f * fz);
    const float c000 = lattice(xi, yi, zi, seed), c100 = lattice(xi + 1, yi, zi, seed);
    const float c010 = lattice(xi, yi + 1, zi, seed), c110 = lattice(xi + 1, yi + 1, zi, seed);
    const float c001 = lattice(xi, yi, zi + 1, seed), c101 = lattice(xi + 1, yi, zi + 1, seed);
    const float c011 = lattice(xi, yi + 1, zi + 1, seed), c111 = lattice(xi + 1, yi + 1, zi + 1, seed);
    const float c00 = c000 + (c100 - c000) * ux;
    const float c10 = c010 + (c110 - c010) * ux;
    const float c01 = c001 + (c101 - c001) * ux;
    const float c11 = c011 + (c111 - c011) * ux;
    const float c0 = c00 + (c10 - c00) * uy;
    const float c1 = c01 + (c11 - c01) * uy;
    return c0 + (c1 - c0) * uz;
}

__host__ __device__ inline double orbital_omega(double mass, double spin, double radius) {
    const double am = fabs(spin);
    const double sm = sqrt(mxd(mass, 1e-12));
    const double sr = sqrt(mxd(radius, 1e-12));
    const double w = sm / (radius * sr + am * sm);
    return (spin < 0.0) ? -w : w;
}

__device__ __forceinline__ double smooth_unit(double x) {
    const double t = cd(x, 0.0, 1.0);
    return t * t * (3.0 - 2.0 * t);
}

// Radiance (out[0..2]) and opacity (out[3]) of the thin disk at (radius,
// azimuth, redshift), AccretionDiskModel::shade (accretion_disk_model.hpp:245-316)
// with the base temperature of the hydro model.
__device__ __noinline__ void disk_radiance(const ShadeDesc& D, double radius_in, double azimuth, double redshift, double* out) {
    const float* P = D.profile;
    const double mass = D.mass;
    const double radius = mxd(radius_in, 1e-9);
    const double inner = D.inner, outer = D.outer;
    double base;
    if (D.hydro_model == 1u) {
        base = pow(mxd(nt_flux(D, radius_in) / D.nt_flux_peak, 0.0), 0.25) * D.nt_rate_factor;
    } else {
        const double u = cd(inner / radius, 1e-4, 1.0);
        base = temperature_shape_d(u, static_cast<double>(P[DP_T_EXPONENT]), static_cast<double>(P[DP_ZERO_TORQUE])) *
               static_cast<double>(P[DP_T_NORMALIZATION]);
    }
    const double soft = mxd(static_cast<double>(P[DP_EDGE_SOFTNESS]), 0.05);
    const double envelope =
        smooth_unit((radius - inner) / (0.8 * soft * mass)) * smooth_unit((outer - radius) / (1.5 * soft * mass));
    const double rotation = static_cast<double>(P[DP_ROTATION]) * D.time;
    double shear_phase = azimuth - orbital_omega(mass, D.disk_spin, radius) * rotation;
    shear_phase -= kTwoPiD * floor(shear_phase / kTwoPiD);
    double pattern_phase = azimuth - D.pattern_omega * rotation;
    pattern_phase -= kTwoPiD * floor(pattern_phase / kTwoPiD);
    const float log_ratio = static_cast<float>(log(mxd(radius / inner, 1.0)));
    const float log_span = mxf(static_cast<float>(log(mxd(outer / inner, 1.0001))), 1e-4f);
    const float radial = log_ratio / log_span;
    const float two_pi_f = 2.0f * 3.14159265358979323846f;
    const float ring_wave = 0.5f + 0.5f * cosf(two_pi_f * P[DP_RING_FREQ] * radial);
    const float ring_sharp = mxf(P[DP_RING_SHARP], 1.0f);
    const float ring = mxf(
        1.0f + P[DP_RING_AMP] * (powf(ring_wave, ring_sharp) * sqrtf(3.14159265358979323846f * ring_sharp) - 1.0f),
        0.0f);
    const float arms = floorf(P[DP_ARMS] + 0.5f);
    const float spiral =
        (arms > 0.5f)
            ? mxf(1.0f + P[DP_SPIRAL_AMP] * cosf(arms * (static_cast<float>(pattern_phase) - P[DP_PITCH] * log_ratio)),
                  0.0f)
            : 1.0f;
    float ss, sc;
    sincosf(static_cast<float>(shear_phase), &ss, &sc);
    int octaves = static_cast<int>(P[DP_TURB_OCTAVES] + 0.5f);
    octaves = octaves < 1 ? 1 : (octaves > 6 ? 6 : octaves);
    const uint32_t seed = static_cast<uint32_t>(mxf(P[DP_NOISE_SEED], 0.0f));
    const float detail = static_cast<float>(cd(D.detail, 0.0, 1.0));
    float total = 0.0f, amp = 1.0f, freq = 1.0f, norm = 0.0f;
    {
        const float nx = log_ratio * P[DP_TURB_SCALE] * P[DP_RADIAL_STRETCH];
        const float ny = sc * P[DP_TURB_SCALE], nz = ss * P[DP_TURB_SCALE];
        for (int o = 0; o < octaves; ++o) {
            total += value_noise(nx * freq, ny * freq, nz * freq, seed + static_cast<uint32_t>(o) * 7919U) * amp;
            norm += amp;
            amp *= 0.5f;
            freq *= 2.0f;
        }
    }
    const float turbulence = expf(1.5f * P[DP_TURB_AMP] * detail * (total / mxf(norm, 1e-5f)));
    const float gn = value_noise(log_ratio * P[DP_GRAIN_SCALE] * P[DP_RADIAL_STRETCH], sc * P[DP_GRAIN_SCALE],
                                 ss * P[DP_GRAIN_SCALE], seed + 104729U);
    const float grain = mxf(1.0f + P[DP_GRAIN_AMP] * detail * gn, 0.0f);
    const float flux_mod = cf(ring * spiral * turbulence * grain, 0.0f, 8.0f);
    const double span = mxd(static_cast<double>(P[DP_PEAK_T]) - static_cast<double>(P[DP_FLOOR_T]), 0.0);
    const double local_t =
        (static_cast<double>(P[DP_FLOOR_T]) + span * base) * pow(mxd(static_cast<double>(flux_mod), 1e-4), 0.25);
    const double g = mxd(redshift, 1e-3);
    double xyz[3];
    planck_xyz(D.lambda_um, D.weight, local_t * g, xyz);
    const double inv = 1.0 / mxd(static_cast<double>(P[DP_REF_LUMINANCE]), 1e-30);
    const double X = xyz[0] * inv, Y = xyz[1] * inv, Z = xyz[2] * inv;
    const double lr = mxd(3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z, 0.0);
    const double lg = mxd(-0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z, 0.0);
    const double lb = mxd(0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z, 0.0);
    const double gain = static_cast<double>(P[DP_BRIGHTNESS]) * pow(g, static_cast<double>(P[DP_BEAMING])) * envelope;
    double red = lr * gain, green = lg * gain, blue = lb * gain;
    const double luma = 0.2126 * red + 0.7152 * green + 0.0722 * blue;
    const double sat = static_cast<double>(P[DP_SATURATION]);
    red = mxd(0.0, luma + (red - luma) * sat);
    green = mxd(0.0, luma + (green - luma) * sat);
    blue = mxd(0.0, luma + (blue - luma) * sat);
    const double ts = static_cast<double>(P[DP_TINT_STRENGTH]);
    red *= 1.0 + (static_cast<double>(P[DP_TINT_R]) - 1.0) * ts;
    green *= 1.0 + (static_cast<double>(P[DP_TINT_G]) - 1.0) * ts;
    blue *= 1.0 + (static_cast<double>(P[DP_TINT_B]) - 1.0) * ts;
    out[0] = static_cast<double>(static_cast<float>(red));
    out[1] = static_cast<double>(static_cast<float>(green));
    out[2] = static_cast<double>(static_cast<float>(blue));
    // opacity of the crossing (accretion_disk_model.hpp:312)
    out[3] = cd(envelope * 0.95 * static_cast<double>(P[DP_OPACITY_SCALE]) *
                    cd(sqrt(fmin(static_cast<double>(flux_mod), 1.0)), 0.15, 1.0),
                0.0, 0.98);
}

// ---- hydro model 2: the Fishbone-Moncrief torus ----
constexpr double kMinThroughputVol = 0.01;  // the reference's loop condition (throughput > 0.01)
// One step's chord through the torus, from and to Boyer-Lindquist points as
// Cartesian (r sin th cos ph, r sin th sin ph, r cos th), for a ray of L_z / E
// = l_over_e: the emission-absorption integral over samples at the chord's
// midpoints within the bounding sphere, sampling_density per M, at most 128
// (HydroDiskContext::integrate_segment, hydro_disk_shading.hpp:173-269), added
// to the ray's gathered light at the throughput left
// (accumulate_fishbone_moncrief_segment, software_compute_engine.hpp:1117-1144).
// A ray gathers nothing once its throughput is 0.01 or less (the reference's
// loop ends there).
__device__ __noinline__ void fm_segment(const ShadeDesc& D, const double* from, const double* to, double l_over_e,
                                        double* V) {
    if (!D.fm_valid) return;
    const bool seen = V[VL_HIT] != 0.0;
    if (seen && !(V[VL_THR] > kMinThroughputVol)) return;
    const double dx = to[0] - from[0], dy = to[1] - from[1], dz = to[2] - from[2];
    const double len2 = dx * dx + dy * dy + dz * dz;
    if (len2 < 1e-24) return;
    const double len = sqrt(len2);
    const double b = (from[0] * dx + from[1] * dy + from[2] * dz) / len2;
    const double c = (from[0] * from[0] + from[1] * from[1] + from[2] * from[2] - D.fm_outer * D.fm_outer) / len2;
    const double disc = b * b - c;
    if (disc <= 0.0) return;
    const double root = sqrt(disc);
    const double t0 = cd(-b - root, 0.0, 1.0), t1 = cd(-b + root, 0.0, 1.0);
    if (t1 <= t0) return;
    const double clipped = len * (t1 - t0);
    const double m = D.fm_m;
    int count = static_cast<int>(ceil(clipped * D.fm_density / m));
    count = count < 1 ? 1 : (count > 128 ? 128 : count);
    const double step = clipped / static_cast<double>(count);
    const float* P = D.profile;
    const double span = mxd(D.fm_h_max - 1.0, 1e-12);
    const double peak_t = static_cast<double>(P[DP_PEAK_T]), floor_t = static_cast<double>(P[DP_FLOOR_T]);
    const double beaming = static_cast<double>(P[DP_BEAMING]), brightness = static_cast<double>(P[DP_BRIGHTNESS]);
    const double inv_ref = 1.0 / mxd(static_cast<double>(P[DP_REF_LUMINANCE]), 1e-30);
    const double sat = static_cast<double>(P[DP_SATURATION]), ts = static_cast<double>(P[DP_TINT_STRENGTH]);
    const torus::Torus T{D.fm_m, D.fm_a, D.fm_rh, D.fm_l, D.fm_w_in};
    double rad[3] = {0.0, 0.0, 0.0}, trans = 1.0, wsum = 0.0, zsum = 0.0;
    for (int i = 0; i < count; ++i) {
        const double t = t0 + (t1 - t0) * ((static_cast<double>(i) + 0.5) / static_cast<double>(count));
        const double px = from[0] + t * dx, py = from[1] + t * dy, pz = from[2] + t * dz;
        const double radius = sqrt(px * px + py * py + pz * pz);
        if (radius < D.fm_inner || radius > D.fm_outer) continue;
        const double theta = acos(cd(pz / radius, -1.0, 1.0));
        const double h = torus::enthalpy(T, radius, theta);
        if (!(h > 1.0 + 1e-9)) continue;
        const double ratio = cd((h - 1.0) / span, 0.0, 1.0);
        const double tau = D.fm_kappa * pow(ratio, D.fm_exponent) * step / m;
        if (tau < 1e-12) continue;
        double ut, uphi;
        torus::four_velocity(T, radius, theta, ut, uphi);
        if (ut <= 1e-12) continue;
        // AccretionDiskModel::redshift_factor (accretion_disk_model.hpp:218-221)
        const double den = ut * (1.0 - (uphi / ut) * l_over_e);
        const double g = (fabs(den) > 1e-9) ? cd(1.0 / den, 0.05, 4.0) : 1.0;
        // blackbody colour of the observed temperature, then the disk profile's grading
        double xyz[3];
        planck_xyz(D.lambda_um, D.weight, (floor_t + (peak_t - floor_t) * ratio) * g, xyz);
        const double X = xyz[0] * inv_ref, Y = xyz[1] * inv_ref, Z = xyz[2] * inv_ref;
        const double gain = brightness * pow(g, beaming);
        double red = mxd(3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z, 0.0) * gain;
        double green = mxd(-0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z, 0.0) * gain;
        double blue = mxd(0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z, 0.0) * gain;
        const double luma = 0.2126 * red + 0.7152 * green + 0.0722 * blue;
        red = mxd(0.0, luma + (red - luma) * sat);
        green = mxd(0.0, luma + (green - luma) * sat);
        blue = mxd(0.0, luma + (blue - luma) * sat);
        red *= 1.0 + (static_cast<double>(P[DP_TINT_R]) - 1.0) * ts;
        green *= 1.0 + (static_cast<double>(P[DP_TINT_G]) - 1.0) * ts;
        blue *= 1.0 + (static_cast<double>(P[DP_TINT_B]) - 1.0) * ts;
        const double st = exp(-tau);
        const double w = trans * (1.0 - st);
        rad[0] += w * red;
        rad[1] += w * green;
        rad[2] += w * blue;
        wsum += w;
        zsum += w * g;
        trans *= st;
        if (trans < 0.002) break;
    }
    const double opacity = 1.0 - trans;
    if (opacity <= 1e-6) return;
    const double thr = seen ? V[VL_THR] : 1.0;
    V[VL_R] += thr * rad[0];
    V[VL_G] += thr * rad[1];
    V[VL_B] += thr * rad[2];
    V[VL_THR] = thr * (1.0 - opacity);
    V[VL_Z] = (wsum > 1e-30) ? (zsum / wsum) : 1.0;
    V[VL_HIT] = 1.0;
}

// ---- translucent-disk continuation ----
// The reference's image path does not end a ray at the disk
// (software_compute_engine.hpp:1660, 1743-1765): each crossing adds the disk's
// radiance at the throughput left and lowers the throughput by the crossing's
// opacity, and the ray goes on while the throughput exceeds 0.01 (the loop
// condition there), to its capture or escape.  The tracers record each
// crossing (cont_record) and the ray's end (cont_finish) and follow a ray for
// at most kMaxCrossings crossings; the shading pass shades the crossings in
// order with the throughput rule, in parallel over rays (shading a crossing
// where it is found would run it one lane at a time while the warp waits).
constexpr double kMinThroughput = 0.01;

__device__ __forceinline__ void cont_record(const ContOut& C, uint64_t o, uint32_t k, double r, double phi,
                                            double g) {
    C.cross[(3 * k) * C.stride + o] = r;
    C.cross[(3 * k + 1) * C.stride + o] = phi;
    C.cross[(3 * k + 2) * C.stride + o] = g;
}

// End of a ray's trace: crossings recorded, its class at the end (UNFINISHED
// also when it stopped at kMaxCrossings) and whether r_last lies inside 3 r_s;
// with the sky on, the sky-lookup direction e at the end.
__device__ __forceinline__ void cont_finish(const ContOut& C, uint64_t o, uint32_t n_cross, uint32_t status,
                                            double r_last, double m, const double* e = nullptr) {
    C.info[o] = n_cross | (status << CI_FATE_SHIFT) | ((r_last < 6.0 * m) ? CI_INSIDE_3RS : 0u);
    if (C.exit && e) {
        C.exit[o] = e[0];
        C.exit[C.stride + o] = e[1];
        C.exit[2 * C.stride + o] = e[2];
    }
}

}  // namespace

}  // namespace relsim
