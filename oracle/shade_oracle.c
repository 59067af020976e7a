/*
 * shade_oracle.c -- CPU oracle of the pixel shading tail (disk colour and
 * tonemapping of GpuPixelOutput).
 *
 * TEST INFRASTRUCTURE ONLY (same rules as ks_oracle.c): a plain-C restatement
 * used as the checker of the CUDA shading pass.
 *
 * What it restates (reference = Wartets/Relativity-Simulator,
 * include/relativistic/...):
 *   - primary disk profile: push-constant overrides and finalize
 *       render/accretion_disk/accretion_disk_model.hpp:180-196
 *   - blackbody colour: Planck radiance on 33 trapezoid nodes over 380-780 nm
 *     against the CIE 1931 colour-matching functions in the multi-lobe Gaussian
 *     fit of Wyman, Sloan & Shirley (JCGT 2013), XYZ -> linear sRGB (IEC
 *     61966-2-1 matrix)   accretion_disk_model.hpp:52-88, 198-203;
 *     optics/cie_observer.hpp:24-88
 *   - thin-disk shading: temperature profile, edge envelope, rings, spiral arms,
 *     value-noise turbulence and grain, Doppler beaming, colour grading, opacity
 *       accretion_disk_model.hpp:90-178, 205-316
 *   - Novikov-Thorne base temperature (hydro model 1): Page-Thorne flux
 *     normalised by its peak over the disk, times accretion_rate_scale^(1/4)
 *       hydro/novikov_thorne.hpp:63-165, 295-325;
 *       render/accretion_disk/hydro_disk_shading.hpp:44-62, 160-171
 *   - tonemapping (clamp, ACES fit of Narkowicz 2015, log luminance, extended
 *     Reinhard) and the sRGB transfer curve
 *       render/software_compute_engine.hpp:3461-3516
 *   - composition of a traced ray's pixel with the procedural sky disabled
 *     (software_compute_engine.hpp:1538-1611): a disk hit contributes the
 *     radiance of its crossing; escaped and captured rays are black.
 * Float and double are used where the reference uses them.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "ks_oracle.h"

#define SH_PI 3.14159265358979323846
#define SH_TWO_PI (2.0 * SH_PI)

static inline double max_d(double a, double b) { return (a < b) ? b : a; }
static inline double min_d(double a, double b) { return (b < a) ? b : a; }
static inline double clamp_d(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
static inline float max_f(float a, float b) { return (a < b) ? b : a; }
static inline float clamp_f(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

/* GpuDiskProfile field order (render/gpu_types.hpp:42-75) */
enum {
    DP_ENABLED = 0, DP_INNER_SCALE, DP_OUTER_UNITS, DP_PEAK_T, DP_FLOOR_T, DP_T_EXPONENT, DP_ZERO_TORQUE, DP_BEAMING,
    DP_BRIGHTNESS, DP_SATURATION, DP_TINT_STRENGTH, DP_OPACITY_SCALE, DP_TINT_R, DP_TINT_G, DP_TINT_B, DP_ROTATION,
    DP_RING_AMP, DP_RING_FREQ, DP_RING_SHARP, DP_ARMS, DP_PITCH, DP_SPIRAL_AMP, DP_TURB_AMP, DP_TURB_SCALE,
    DP_TURB_OCTAVES, DP_RADIAL_STRETCH, DP_GRAIN_AMP, DP_GRAIN_SCALE, DP_REF_LUMINANCE, DP_NOISE_SEED,
    DP_T_NORMALIZATION, DP_EDGE_SOFTNESS
};

/* ---- colour ------------------------------------------------------------ */
static double lobe(double x, double alpha, double mu, double s1, double s2)
{
    const double s = (x < mu) ? s1 : s2;
    const double t = (x - mu) / s;
    return alpha * exp(-0.5 * t * t);
}
static double cie_x(double l) { return lobe(l, 1.056, 599.8, 37.9, 31.0) + lobe(l, 0.362, 442.0, 16.0, 26.7) - lobe(l, 0.065, 501.1, 20.4, 26.2); }
static double cie_y(double l) { return lobe(l, 0.821, 568.8, 46.9, 40.5) + lobe(l, 0.286, 530.9, 16.3, 31.1); }
static double cie_z(double l) { return lobe(l, 1.217, 437.0, 11.8, 36.0) + lobe(l, 0.681, 459.0, 26.0, 13.8); }

#define N_SPECTRAL 32
void orc_planck_xyz(double temperature_k, double xyz[3])
{
    const double step = (780.0 - 380.0) / (double)N_SPECTRAL;
    const double t = clamp_d(temperature_k, 300.0, 400000.0);
    xyz[0] = xyz[1] = xyz[2] = 0.0;
    for (int i = 0; i <= N_SPECTRAL; ++i) {
        const double lnm = 380.0 + (double)i * step;
        const double trap = (i == 0 || i == N_SPECTRAL) ? 0.5 : 1.0;
        const double lum = lnm * 1e-3;
        const double e = 14387.76877 / (lum * t); /* second radiation constant, um K */
        if (e > 80.0) continue;
        const double l2 = lum * lum;
        const double rad = 1.0 / (l2 * l2 * lum * expm1(e));
        xyz[0] += rad * (trap * cie_x(lnm));
        xyz[1] += rad * (trap * cie_y(lnm));
        xyz[2] += rad * (trap * cie_z(lnm));
    }
}

void orc_blackbody_rgb(double temperature_k, double reference_luminance, double rgb[3])
{
    double xyz[3];
    orc_planck_xyz(temperature_k, xyz);
    const double inv = 1.0 / max_d(reference_luminance, 1e-30);
    const double X = xyz[0] * inv, Y = xyz[1] * inv, Z = xyz[2] * inv;
    rgb[0] = max_d(3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z, 0.0);
    rgb[1] = max_d(-0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z, 0.0);
    rgb[2] = max_d(0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z, 0.0);
}

/* ---- profile ------------------------------------------------------------ */
static double temperature_shape(double u, double exponent, double zero_torque)
{
    const double boundary = max_d(1.0 - zero_torque * sqrt(u), 0.0);
    return pow(u, exponent) * pow(boundary, 0.25);
}

static double temperature_shape_peak(double exponent, double zero_torque)
{
    double lo = 1e-4, hi = 1.0;
    for (int it = 0; it < 48; ++it) { /* ternary search on a unimodal shape */
        const double a = lo + (hi - lo) / 3.0;
        const double b = hi - (hi - lo) / 3.0;
        if (temperature_shape(a, exponent, zero_torque) < temperature_shape(b, exponent, zero_torque)) lo = a;
        else hi = b;
    }
    return max_d(temperature_shape(0.5 * (lo + hi), exponent, zero_torque), temperature_shape(1.0, exponent, zero_torque));
}

void orc_resolve_profile(const float in[32], const double overrides[4], float out[32])
{
    memcpy(out, in, sizeof(float) * 32);
    out[DP_PEAK_T] = (float)overrides[0];
    out[DP_FLOOR_T] = (float)overrides[1];
    out[DP_SATURATION] = (float)overrides[2];
    out[DP_BEAMING] = (float)overrides[3];
    out[DP_PEAK_T] = clamp_f(out[DP_PEAK_T], 1000.0f, 200000.0f);
    out[DP_FLOOR_T] = clamp_f(out[DP_FLOOR_T], 0.0f, out[DP_PEAK_T]);
    const double peak = temperature_shape_peak((double)out[DP_T_EXPONENT], (double)out[DP_ZERO_TORQUE]);
    out[DP_T_NORMALIZATION] = (float)(1.0 / max_d(peak, 1e-6));
    double xyz[3];
    orc_planck_xyz((double)out[DP_PEAK_T], xyz);
    out[DP_REF_LUMINANCE] = (float)max_d(xyz[1], 1e-30);
}

/* ---- Novikov-Thorne ------------------------------------------------------ */
typedef struct { double m, a_star, x0, x1, x2, x3, r_isco; } nt_disk;

static void nt_init(nt_disk* d, double mass, double spin)
{
    d->m = mass;
    d->a_star = clamp_d(spin / mass, -0.999999999, 0.999999999);
    const double a = d->a_star;
    const double z1 = 1.0 + cbrt(1.0 - a * a) * (cbrt(1.0 + a) + cbrt(1.0 - a));
    const double z2 = sqrt(3.0 * a * a + z1 * z1);
    const double root = sqrt(max_d(0.0, (3.0 - z1) * (3.0 + z1 + 2.0 * z2)));
    d->r_isco = mass * ((a >= 0.0) ? (3.0 + z2 - root) : (3.0 + z2 + root));
    d->x0 = sqrt(d->r_isco / mass);
    const double psi = acos(clamp_d(a, -1.0, 1.0)) / 3.0;
    d->x1 = 2.0 * cos(psi - SH_PI / 3.0);
    d->x2 = 2.0 * cos(psi + SH_PI / 3.0);
    d->x3 = -2.0 * cos(psi);
}

/* Page & Thorne (1974) flux integral f(x), x = sqrt(r / M). */
static double page_thorne_f(const nt_disk* d, double x)
{
    if (x < d->x0) return 0.0;
    const double a = d->a_star, x0 = d->x0, x1 = d->x1, x2 = d->x2, x3 = d->x3;
    double f = x - x0;
    if (fabs(a) > 1e-15) f -= 1.5 * a * log(x / x0);
    {
        const double c = 3.0 * (x1 - a) * (x1 - a) / (x1 * (x1 - x2) * (x1 - x3));
        f -= c * log(max_d((x - x1) / (x0 - x1), 1e-30));
    }
    if (fabs(x2) > 1e-12) {
        const double c = 3.0 * (x2 - a) * (x2 - a) / (x2 * (x2 - x1) * (x2 - x3));
        f -= c * log(max_d((x - x2) / (x0 - x2), 1e-30));
    }
    {
        const double c = 3.0 * (x3 - a) * (x3 - a) / (x3 * (x3 - x1) * (x3 - x2));
        f -= c * log(max_d((x - x3) / (x0 - x3), 1e-30));
    }
    return max_d(0.0, f);
}

static double nt_flux(const nt_disk* d, double r)
{
    if (r < d->r_isco) return 0.0;
    const double x = sqrt(r / d->m);
    const double x3 = x * x * x;
    const double den = x * (x3 + d->a_star);
    if (den <= 1e-24) return 0.0;
    const double factor = (3.0 * d->m * 1.0) / (8.0 * SH_PI * (r * r * r));
    return max_d(0.0, factor * (page_thorne_f(d, x) / den));
}

/* Peak flux over the disk (192 log-spaced radii) and rate^(1/4). */
void orc_nt_context(double mass, double spin, double inner, double outer, float accretion_rate_scale, double out[2])
{
    const double m = max_d(mass, 1e-9);
    const double a = clamp_d(spin, -0.999 * m, 0.999 * m);
    const double in_r = max_d(inner, 1e-9);
    const double out_r = max_d(outer, in_r * 1.0001);
    nt_disk d;
    nt_init(&d, m, a);
    const double lo = max_d(in_r, d.r_isco * 1.0001);
    const double hi = max_d(out_r, lo * 1.01);
    const double ratio = hi / lo;
    double peak = 0.0;
    for (int i = 0; i < 192; ++i) {
        const double frac = (double)i / 191.0;
        peak = max_d(peak, nt_flux(&d, lo * pow(ratio, frac)));
    }
    out[0] = (peak > 1e-300) ? peak : 1.0;
    out[1] = pow(max_d((double)accretion_rate_scale, 1e-6), 0.25);
}

/* ---- procedural modulation ---------------------------------------------- */
static uint32_t lowbias32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

static float lattice(int32_t x, int32_t y, int32_t z, uint32_t seed)
{
    const uint32_t h = (uint32_t)x * 374761393U + (uint32_t)y * 668265263U + (uint32_t)z * 2147483647U + seed * 1274126177U;
    return (float)(lowbias32(h) & 0x00FFFFFFU) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
}

static float value_noise(float x, float y, float z, uint32_t seed)
{
    const float fx0 = floorf(x), fy0 = floorf(y), fz0 = floorf(z);
    const int32_t xi = (int32_t)fx0, yi = (int32_t)fy0, zi = (int32_t)fz0;
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

static float fractal_noise(float x, float y, float z, int octaves, uint32_t seed)
{
    float total = 0.0f, amp = 1.0f, freq = 1.0f, norm = 0.0f;
    for (int o = 0; o < octaves; ++o) {
        total += value_noise(x * freq, y * freq, z * freq, seed + (uint32_t)o * 7919U) * amp;
        norm += amp;
        amp *= 0.5f;
        freq *= 2.0f;
    }
    return total / max_f(norm, 1e-5f);
}

static double smooth_unit(double x)
{
    const double t = clamp_d(x, 0.0, 1.0);
    return t * t * (3.0 - 2.0 * t);
}

static double reduce_angle(double a) { return a - SH_TWO_PI * floor(a / SH_TWO_PI); }

/* Keplerian angular velocity of a circular equatorial orbit (accretion_disk_model.hpp:205-216). */
static double orbital_omega(double mass, double spin, double radius)
{
    const double am = fabs(spin);
    const double sm = sqrt(max_d(mass, 1e-12));
    const double sr = sqrt(max_d(radius, 1e-12));
    const double w = sm / (radius * sr + am * sm);
    return (spin < 0.0) ? -w : w;
}

/* point: mass, spin, inner, outer, radius, azimuth, redshift, time, detail;
 * base_temperature < 0: the procedural profile.  out: r, g, b, opacity. */
static void shade_point(const float* P, const double* pt, double base_temperature, double out[4])
{
    const double mass = max_d(pt[0], 1e-9);
    const double spin = pt[1];
    const double radius = max_d(pt[4], 1e-9);
    const double inner = max_d(pt[2], 1e-9);
    const double outer = max_d(pt[3], inner * 1.0001);
    const double u = clamp_d(inner / radius, 1e-4, 1.0);
    const double base = (base_temperature >= 0.0)
                            ? base_temperature
                            : temperature_shape(u, (double)P[DP_T_EXPONENT], (double)P[DP_ZERO_TORQUE]) *
                                  (double)P[DP_T_NORMALIZATION];
    const double soft = max_d((double)P[DP_EDGE_SOFTNESS], 0.05);
    const double envelope = smooth_unit((radius - inner) / (0.8 * soft * mass)) * smooth_unit((outer - radius) / (1.5 * soft * mass));
    const double rotation = (double)P[DP_ROTATION] * pt[7];
    const double shear_phase = reduce_angle(pt[5] - orbital_omega(mass, spin, radius) * rotation);
    const double pattern_phase = reduce_angle(pt[5] - orbital_omega(mass, spin, sqrt(inner * outer)) * rotation);
    const float log_ratio = (float)log(max_d(radius / inner, 1.0));
    const float log_span = max_f((float)log(max_d(outer / inner, 1.0001)), 1e-4f);
    const float radial = log_ratio / log_span;
    const float two_pi_f = 2.0f * 3.14159265358979323846f;
    const float ring_wave = 0.5f + 0.5f * cosf(two_pi_f * P[DP_RING_FREQ] * radial);
    const float ring_sharp = max_f(P[DP_RING_SHARP], 1.0f);
    const float ring = max_f(1.0f + P[DP_RING_AMP] * (powf(ring_wave, ring_sharp) * sqrtf(3.14159265358979323846f * ring_sharp) - 1.0f), 0.0f);
    const float arms = floorf(P[DP_ARMS] + 0.5f);
    const float spiral = (arms > 0.5f) ? max_f(1.0f + P[DP_SPIRAL_AMP] * cosf(arms * ((float)pattern_phase - P[DP_PITCH] * log_ratio)), 0.0f) : 1.0f;
    const float sc = cosf((float)shear_phase);
    const float ss = sinf((float)shear_phase);
    int octaves = (int)(P[DP_TURB_OCTAVES] + 0.5f);
    octaves = octaves < 1 ? 1 : (octaves > 6 ? 6 : octaves);
    const uint32_t seed = (uint32_t)max_f(P[DP_NOISE_SEED], 0.0f);
    const float detail = (float)clamp_d(pt[8], 0.0, 1.0);
    const float tn = fractal_noise(log_ratio * P[DP_TURB_SCALE] * P[DP_RADIAL_STRETCH], sc * P[DP_TURB_SCALE], ss * P[DP_TURB_SCALE], octaves, seed);
    const float turbulence = expf(1.5f * P[DP_TURB_AMP] * detail * tn);
    const float gn = value_noise(log_ratio * P[DP_GRAIN_SCALE] * P[DP_RADIAL_STRETCH], sc * P[DP_GRAIN_SCALE], ss * P[DP_GRAIN_SCALE], seed + 104729U);
    const float grain = max_f(1.0f + P[DP_GRAIN_AMP] * detail * gn, 0.0f);
    const float flux_mod = clamp_f(ring * spiral * turbulence * grain, 0.0f, 8.0f);
    const double span = max_d((double)P[DP_PEAK_T] - (double)P[DP_FLOOR_T], 0.0);
    const double local_t = ((double)P[DP_FLOOR_T] + span * base) * pow(max_d((double)flux_mod, 1e-4), 0.25);
    const double g = max_d(pt[6], 1e-3);
    double lin[3];
    orc_blackbody_rgb(local_t * g, (double)P[DP_REF_LUMINANCE], lin);
    const double gain = (double)P[DP_BRIGHTNESS] * pow(g, (double)P[DP_BEAMING]) * envelope;
    /* colour grading (accretion_disk_model.hpp:227-243) */
    double red = lin[0] * gain, green = lin[1] * gain, blue = lin[2] * gain;
    const double luma = 0.2126 * red + 0.7152 * green + 0.0722 * blue;
    const double sat = (double)P[DP_SATURATION];
    red = max_d(0.0, luma + (red - luma) * sat);
    green = max_d(0.0, luma + (green - luma) * sat);
    blue = max_d(0.0, luma + (blue - luma) * sat);
    const double ts = (double)P[DP_TINT_STRENGTH];
    red *= 1.0 + ((double)P[DP_TINT_R] - 1.0) * ts;
    green *= 1.0 + ((double)P[DP_TINT_G] - 1.0) * ts;
    blue *= 1.0 + ((double)P[DP_TINT_B] - 1.0) * ts;
    out[0] = (double)(float)red;
    out[1] = (double)(float)green;
    out[2] = (double)(float)blue;
    out[3] = clamp_d(envelope * 0.95 * (double)P[DP_OPACITY_SCALE] * clamp_d(sqrt(min_d((double)flux_mod, 1.0)), 0.15, 1.0), 0.0, 0.98);
}

void orc_disk_shade(const float profile[32], const double point[9], uint32_t hydro_model, float accretion_rate_scale,
                    double out[4])
{
    double base = -1.0;
    if (hydro_model == 1u) {
        double ctx[2];
        orc_nt_context(point[0], point[1], point[2], point[3], accretion_rate_scale, ctx);
        const double m = max_d(point[0], 1e-9);
        nt_disk d;
        nt_init(&d, m, clamp_d(point[1], -0.999 * m, 0.999 * m));
        base = pow(max_d(nt_flux(&d, point[4]) / ctx[0], 0.0), 0.25) * ctx[1];
    }
    shade_point(profile, point, base, out);
}

static float to_srgb(double v)
{
    if (v <= 0.0031308) return (float)(12.92 * v);
    return (float)(1.055 * pow(v, 1.0 / 2.4) - 0.055);
}

static double aces(double x) { return clamp_d((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0, 1.0); }

void orc_tonemap(const double rgb[3], uint32_t mode, double exposure_ev, float out[3])
{
    const double k = exp2(exposure_ev);
    double r = max_d(0.0, rgb[0] * k), g = max_d(0.0, rgb[1] * k), b = max_d(0.0, rgb[2] * k);
    if (mode == 1u) {
        r = aces(r);
        g = aces(g);
        b = aces(b);
    } else if (mode == 2u) {
        const double lum = 0.2126 * r + 0.7152 * g + 0.0722 * b;
        if (lum > 0.0) {
            const double mapped = log10(1.0 + lum * 100.0) / log10(1.0 + 10000.0);
            const double s = clamp_d(mapped / lum, 0.0, 1.0);
            r = clamp_d(r * s, 0.0, 1.0);
            g = clamp_d(g * s, 0.0, 1.0);
            b = clamp_d(b * s, 0.0, 1.0);
        }
    } else if (mode == 3u) {
        r = (r * (1.0 + r / 25.0)) / (1.0 + r);
        g = (g * (1.0 + g / 25.0)) / (1.0 + g);
        b = (b * (1.0 + b / 25.0)) / (1.0 + b);
    } else {
        r = clamp_d(r, 0.0, 1.0);
        g = clamp_d(g, 0.0, 1.0);
        b = clamp_d(b, 0.0, 1.0);
    }
    out[0] = to_srgb(r);
    out[1] = to_srgb(g);
    out[2] = to_srgb(b);
}

/* Pixel colour of a traced ray (sky disabled): a disk hit is shaded at
 * (r_hit, phi, g) on the camera's disk; every other ray is black.  disk_spin
 * is the clamped spin, inner/outer the disk radii, detail the turbulence
 * anti-aliasing factor of the camera. */
void orc_shade_pixel(const float resolved_profile[32], uint32_t hydro_model, float accretion_rate_scale,
                     uint32_t tonemap_mode, double exposure_ev, double mass, double disk_spin, double inner,
                     double outer, double time, double detail, uint32_t status, double r_hit, double phi, double g,
                     float out[3])
{
    double accum[3] = {0.0, 0.0, 0.0};
    if (status == ORC_RAY_DISK) {
        const double pt[9] = {mass, disk_spin, inner, outer, r_hit, phi, g, time, detail};
        double s[4];
        orc_disk_shade(resolved_profile, pt, hydro_model, accretion_rate_scale, s);
        accum[0] = s[0];
        accum[1] = s[1];
        accum[2] = s[2];
    }
    orc_tonemap(accum, tonemap_mode, exposure_ev, out);
}

/* Pixel colour of a ray followed through the translucent disk
 * (software_compute_engine.hpp:1743-1765, 1777-1795; sky disabled): each
 * recorded crossing k adds the disk's radiance at the throughput left,
 * T_k = prod_{j<k} (1 - opacity_j), while T > 0.01 (the reference's loop
 * condition); with the sky disabled the ray's end adds nothing. */
void orc_shade_cont(const float resolved_profile[32], uint32_t hydro_model, float accretion_rate_scale,
                    uint32_t tonemap_mode, double exposure_ev, double mass, double disk_spin, double inner,
                    double outer, double time, double detail, uint32_t n_cross, const double* cross_r,
                    const double* cross_phi, const double* cross_g, float out[3])
{
    double accum[3] = {0.0, 0.0, 0.0};
    double throughput = 1.0;
    for (uint32_t k = 0; k < n_cross && throughput > 0.01; ++k) {
        const double pt[9] = {mass, disk_spin, inner, outer, cross_r[k], cross_phi[k], cross_g[k], time, detail};
        double sh[4];
        orc_disk_shade(resolved_profile, pt, hydro_model, accretion_rate_scale, sh);
        accum[0] += throughput * sh[0];
        accum[1] += throughput * sh[1];
        accum[2] += throughput * sh[2];
        throughput *= 1.0 - sh[3];
    }
    orc_tonemap(accum, tonemap_mode, exposure_ev, out);
}

/* ---- hydro model 2: the Fishbone-Moncrief torus ------------------------
 * Restated from hydro/fishbone_moncrief.hpp (the Fishbone & Moncrief 1976
 * constant-l torus, G = c = 1) and render/accretion_disk/hydro_disk_shading.hpp
 * (HydroDiskContext::build_torus :76-110, integrate_segment :173-269). */
static double fm_horizon(double m, double a)
{
    const double d = m * m - a * a;
    return (d < 0.0) ? m : m + sqrt(d);
}

static double fm_keplerian_l(double m, double a, double rh, double r) /* fishbone_moncrief.hpp:98-116 */
{
    const double rs = max_d(r, 1.001 * rh);
    const double sm = sqrt(m), sr = sqrt(rs);
    const double num = sm * (rs * rs - 2.0 * a * sm * sr + a * a);
    const double den = rs * sr - 2.0 * m * sr + a * sm;
    return (fabs(den) < 1e-30) ? 0.0 : num / den;
}

static double fm_potential(const orc_fm* t, double r, double theta) /* :118-150 */
{
    if (r <= t->rh * 1.0001) return 1e30;
    const double st = sin(theta), ct = cos(theta);
    const double s2 = max_d(st * st, 1e-30), c2 = ct * ct;
    const double r2 = r * r, a2 = t->a * t->a;
    const double rho2 = r2 + a2 * c2;
    const double delta = r2 - 2.0 * t->m * r + a2;
    const double sigma = (r2 + a2) * (r2 + a2) - a2 * delta * s2;
    const double den = sigma * s2 - 4.0 * t->m * r * t->a * t->l * s2 - t->l * t->l * (delta - a2 * s2);
    if (den <= 0.0 || delta <= 0.0) return 1e30;
    return 0.5 * log(max_d((rho2 * delta * s2) / den, 1e-30));
}

static double fm_enthalpy(const orc_fm* t, double r, double theta) /* :152-159 */
{
    const double w = fm_potential(t, r, theta);
    if (w >= t->w_in) return 1.0;
    return max_d(1.0, exp(t->w_in - w));
}

/* u^t, u^phi of the fluid (:210-224) with the Boyer-Lindquist Kerr inverse
 * metric (metrics/kerr.hpp:151-177). */
static void fm_four_velocity(const orc_fm* t, double r, double theta, double* ut, double* uphi)
{
    const double w = fm_potential(t, r, theta);
    if (w >= 1e20) {
        *ut = 1.0;
        *uphi = 0.0;
        return;
    }
    const double lt = -exp(w), lphi = -t->l * lt;
    const double rr = max_d(r, 1e-12);
    const double st = sin(theta), ct = cos(theta);
    const double s2 = max_d(st * st, 1e-30), c2 = ct * ct;
    const double a2 = t->a * t->a, r2 = rr * rr;
    const double rho2 = r2 + a2 * c2;
    const double delta = r2 - 2.0 * t->m * rr + a2;
    const double sigma = (r2 + a2) * (r2 + a2) - a2 * delta * s2;
    const double gtt = -sigma / (rho2 * delta);
    const double gtp = -(2.0 * t->m * rr * t->a) / (rho2 * delta);
    const double gpp = (delta - a2 * s2) / (rho2 * delta * s2);
    *ut = gtt * lt + gtp * lphi;
    *uphi = gtp * lt + gpp * lphi;
}

void orc_fm_context(double mass, double spin, double r_in_units, double r_center_units, double gamma,
                    double optical_depth_scale, double sampling_density, const float resolved_profile[32], orc_fm* out)
{
    memset(out, 0, sizeof *out);
    memcpy(out->profile, resolved_profile, sizeof out->profile);
    /* the settings are floats in GpuHydroDiskProfile */
    r_in_units = (double)(float)r_in_units;
    r_center_units = (double)(float)r_center_units;
    gamma = (double)(float)gamma;
    optical_depth_scale = (double)(float)optical_depth_scale;
    sampling_density = (double)(float)sampling_density;
    const double m = max_d(mass, 1e-9);
    const double a = clamp_d(spin, -0.999 * m, 0.999 * m);
    out->m = m;
    out->a = a;
    out->rh = fm_horizon(m, a);
    const double r_c = (r_center_units * m > 0.0) ? r_center_units * m : 12.0 * m;
    const double r_in = (r_in_units * m > 0.0) ? r_in_units * m : 6.0 * m;
    const double half_pi = 0.5 * SH_PI;
    out->l = fm_keplerian_l(m, a, out->rh, r_c);
    out->w_in = fm_potential(out, r_in, half_pi);
    const double w_center = fm_potential(out, r_c, half_pi);
    out->h_max = exp(max_d(0.0, out->w_in - w_center));
    out->valid = isfinite(out->h_max) && out->h_max > 1.0 + 1e-9;
    out->inner = 0.8 * r_in;
    out->exponent = 1.0 / max_d(gamma - 1.0, 1e-3);
    out->kappa = optical_depth_scale * max_d((double)resolved_profile[DP_OPACITY_SCALE], 0.0);
    out->density = max_d(sampling_density, 0.1);
    if (!out->valid) return;
    const double step = 0.25 * r_c, limit = 200.0 * r_c;
    double inside = r_c, outside = r_c;
    int found = 0;
    while (outside < limit) {
        outside += step;
        if (!(fm_potential(out, outside, half_pi) < out->w_in)) {
            found = 1;
            break;
        }
        inside = outside;
    }
    if (found) {
        for (int it = 0; it < 48; ++it) {
            const double mid = 0.5 * (inside + outside);
            if (fm_potential(out, mid, half_pi) < out->w_in) inside = mid;
            else outside = mid;
        }
        out->outer = 1.05 * outside;
    } else {
        out->outer = limit;
    }
    out->closed = (uint32_t)found;
}

void orc_fm_segment(const orc_fm* t, const double from[3], const double to[3], double l_over_e, double out[5])
{
    out[0] = out[1] = out[2] = out[3] = 0.0;
    out[4] = 1.0;
    if (!t->valid) return;
    const double dx = to[0] - from[0], dy = to[1] - from[1], dz = to[2] - from[2];
    const double len2 = dx * dx + dy * dy + dz * dz;
    if (len2 < 1e-24) return;
    const double len = sqrt(len2);
    const double b = (from[0] * dx + from[1] * dy + from[2] * dz) / len2;
    const double c = (from[0] * from[0] + from[1] * from[1] + from[2] * from[2] - t->outer * t->outer) / len2;
    const double disc = b * b - c;
    if (disc <= 0.0) return;
    const double root = sqrt(disc);
    const double t0 = clamp_d(-b - root, 0.0, 1.0), t1 = clamp_d(-b + root, 0.0, 1.0);
    if (t1 <= t0) return;
    const double clipped = len * (t1 - t0);
    int count = (int)ceil(clipped * t->density / t->m);
    count = count < 1 ? 1 : (count > 128 ? 128 : count);
    const double step = clipped / (double)count;
    const float* P = t->profile;
    const double span = max_d(t->h_max - 1.0, 1e-12);
    double trans = 1.0, wsum = 0.0, zsum = 0.0;
    for (int i = 0; i < count; ++i) {
        const double u = t0 + (t1 - t0) * (((double)i + 0.5) / (double)count);
        const double px = from[0] + u * dx, py = from[1] + u * dy, pz = from[2] + u * dz;
        const double radius = sqrt(px * px + py * py + pz * pz);
        if (radius < t->inner || radius > t->outer) continue;
        const double theta = acos(clamp_d(pz / radius, -1.0, 1.0));
        const double h = fm_enthalpy(t, radius, theta);
        if (!(h > 1.0 + 1e-9)) continue;
        const double ratio = clamp_d((h - 1.0) / span, 0.0, 1.0);
        const double tau = t->kappa * pow(ratio, t->exponent) * step / t->m;
        if (tau < 1e-12) continue;
        double ut, uphi;
        fm_four_velocity(t, radius, theta, &ut, &uphi);
        if (ut <= 1e-12) continue;
        /* AccretionDiskModel::redshift_factor (accretion_disk_model.hpp:218-221) */
        const double den = ut * (1.0 - (uphi / ut) * l_over_e);
        const double g = (fabs(den) > 1e-9) ? clamp_d(1.0 / den, 0.05, 4.0) : 1.0;
        double lin[3];
        orc_blackbody_rgb(((double)P[DP_FLOOR_T] + ((double)P[DP_PEAK_T] - (double)P[DP_FLOOR_T]) * ratio) * g,
                          (double)P[DP_REF_LUMINANCE], lin);
        const double gain = (double)P[DP_BRIGHTNESS] * pow(g, (double)P[DP_BEAMING]);
        double red = lin[0] * gain, green = lin[1] * gain, blue = lin[2] * gain;
        const double luma = 0.2126 * red + 0.7152 * green + 0.0722 * blue;
        const double sat = (double)P[DP_SATURATION];
        red = max_d(0.0, luma + (red - luma) * sat);
        green = max_d(0.0, luma + (green - luma) * sat);
        blue = max_d(0.0, luma + (blue - luma) * sat);
        const double ts = (double)P[DP_TINT_STRENGTH];
        red *= 1.0 + ((double)P[DP_TINT_R] - 1.0) * ts;
        green *= 1.0 + ((double)P[DP_TINT_G] - 1.0) * ts;
        blue *= 1.0 + ((double)P[DP_TINT_B] - 1.0) * ts;
        const double st = exp(-tau);
        const double w = trans * (1.0 - st);
        out[0] += w * red;
        out[1] += w * green;
        out[2] += w * blue;
        wsum += w;
        zsum += w * g;
        trans *= st;
        if (trans < 0.002) break;
    }
    out[3] = 1.0 - trans;
    out[4] = (wsum > 1e-30) ? (zsum / wsum) : 1.0;
}

/* accumulate_fishbone_moncrief_segment (software_compute_engine.hpp:1117-1144)
 * into a ray's gathered light vol[6] (r, g, b, throughput, redshift, seen),
 * all 0 before its first emitting segment; nothing once the throughput is
 * 0.01 or less (the reference's loop ends there). */
void orc_fm_accumulate(const orc_fm* t, const double from[3], const double to[3], double l_over_e, double vol[6])
{
    const int seen = vol[5] != 0.0;
    if (seen && !(vol[3] > 0.01)) return;
    double s[5];
    orc_fm_segment(t, from, to, l_over_e, s);
    if (s[3] <= 1e-6) return;
    const double thr = seen ? vol[3] : 1.0;
    vol[0] += thr * s[0];
    vol[1] += thr * s[1];
    vol[2] += thr * s[2];
    vol[3] = thr * (1.0 - s[3]);
    vol[4] = s[4];
    vol[5] = 1.0;
}
