// rt_shade.cu -- pixel shading pass (GpuPixelOutput's colour) for sm_100a.
//
// After a trace, one thread per ray turns the record (class, r_hit, phi, g)
// into the pixel's sRGB colour, as the reference's CPU image path does
// (software_compute_engine.hpp:1538-1611): a disk hit is shaded as the thin
// disk at the crossing (AccretionDiskModel::shade,
// render/accretion_disk/accretion_disk_model.hpp:245-316, with the
// Novikov-Thorne base temperature of hydro model 1,
// render/accretion_disk/hydro_disk_shading.hpp:160-171) and the accumulated
// radiance is tonemapped (apply_tonemapping, :3461-3516).  The procedural sky
// is not part of this library, so escaped and captured rays are black.  The
// tracers stop at the first disk crossing; the reference continues through a
// semi-transparent disk (opacity <= 0.98) and adds later crossings at the
// remaining throughput, which is not done here.
//
// Per-camera constants (the resolved profile, the Novikov-Thorne flux
// normalisation, the spectral table of the blackbody colour) are computed on
// the host; the same helpers run on both sides.  Float is used where the
// reference uses float (the pattern and noise), double elsewhere.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "rt_internal.h"

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

// CIE 1931 colour-matching functions, multi-lobe Gaussian fit (Wyman, Sloan &
// Shirley, JCGT 2013), as optics/cie_observer.hpp:24-45 uses them.
double lobe(double x, double alpha, double mu, double s1, double s2) {
    const double s = (x < mu) ? s1 : s2;
    const double t = (x - mu) / s;
    return alpha * std::exp(-0.5 * t * t);
}

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

double temperature_shape(double u, double exponent, double zero_torque) {
    const double boundary = mxd(1.0 - zero_torque * std::sqrt(u), 0.0);
    return std::pow(u, exponent) * std::pow(boundary, 0.25);
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

__device__ __forceinline__ float to_srgb(double v) {
    if (v <= 0.0031308) return static_cast<float>(12.92 * v);
    return static_cast<float>(1.055 * pow(v, 1.0 / 2.4) - 0.055);
}

__device__ __forceinline__ double aces(double x) {
    return cd((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0, 1.0);
}

// Radiance of the thin disk at (radius, azimuth, redshift), AccretionDiskModel::shade
// (accretion_disk_model.hpp:245-316) with the base temperature of the hydro model.
__device__ void disk_radiance(const ShadeDesc& D, double radius_in, double azimuth, double redshift, double* out) {
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
}

__global__ void __launch_bounds__(256) shade_kernel(const ShadeDesc* __restrict__ Dp,
                                                    const uint32_t* __restrict__ status,
                                                    const double* __restrict__ r_hit,
                                                    const double* __restrict__ phi,
                                                    const double* __restrict__ g, rt_pixel_out* __restrict__ pixels,
                                                    uint64_t n) {
    const ShadeDesc& D = *Dp;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        double acc[3] = {0.0, 0.0, 0.0};
        if (status[i] == RT_RAY_DISK) disk_radiance(D, r_hit[i], phi[i], g[i], acc);
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
    if (s.hydro_model > 1u || s.sky_enabled != 0u || s.tonemapping_mode > 3u) return false;
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
    return true;
}

void launch_shade(const ShadeDesc* desc, const uint32_t* status, const double* r_hit, const double* phi,
                  const double* g, rt_pixel_out* pixels, uint64_t n, void* stream) {
    if (n == 0) return;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    shade_kernel<<<static_cast<unsigned>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(desc, status, r_hit,
                                                                                                phi, g, pixels, n);
}

}  // namespace relsim
