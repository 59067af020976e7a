// rt_sky.cuh -- the procedural sky (SkyboxRenderer::sample_procedural_sky,
// render/skybox_renderer.hpp:1594-1672) as host/device code: the sky colour
// behind an escaped ray from its exit direction.
//
// Layers, in the reference's order: background, volumetric nebulae (three
// fBm emission fields per layer over a galactic-plane and asymmetry
// envelope, curl-displaced, with ridged-noise absorption), interstellar dust,
// galaxies (six morphologies on an equal-area ring/sector partition), star
// clusters (Plummer halo and members), quasars with Doppler-boosted jets,
// pulsars with swept beams and wind nebulae, supernova remnants, stars on a
// hashed 3-D grid with eight point-spread models and six placement models;
// master intensity, hue/saturation, then the celestial grid.  The settings
// are the GpuSkyProfile image (rt_sky_profile.h).  Every step follows the
// reference's arithmetic and types (float where it uses float), so the host
// build matches it to rounding and the device build to the libraries'
// transcendental functions.  The procedural panoramas of the reference (image
// files) are not part of this library.
#pragma once

#include <cmath>
#include <cstdint>

#include "rt_sky_profile.h"

#ifdef __CUDACC__
#define RT_SKY_HD __host__ __device__ __forceinline__
#define RT_SKY_HD_NOINLINE __host__ __device__ __noinline__
#else
#define RT_SKY_HD inline
#define RT_SKY_HD_NOINLINE inline
#endif

namespace relsim {
namespace sky {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kHalfPi = 0.5 * kPi;
constexpr double kDegToRad = kPi / 180.0;

// The double-precision library functions the layers call, each compiled once on
// the device: inlined at their many call sites they made the sky's code larger
// than the instruction cache, and warps in different layers stalled on
// instruction fetch.  Same functions, same results.
#ifdef __CUDACC__
#define RT_SKY_MATH __host__ __device__ __noinline__
#else
#define RT_SKY_MATH inline
#endif
RT_SKY_MATH double m_exp(double x) { return ::exp(x); }
RT_SKY_MATH double m_pow(double x, double y) { return ::pow(x, y); }
RT_SKY_MATH double m_sin(double x) { return ::sin(x); }
RT_SKY_MATH double m_cos(double x) { return ::cos(x); }
RT_SKY_MATH double m_atan2(double y, double x) { return ::atan2(y, x); }
RT_SKY_MATH double m_log(double x) { return ::log(x); }
RT_SKY_MATH double m_remainder(double x, double y) { return ::remainder(x, y); }
RT_SKY_MATH double m_fmod(double x, double y) { return ::fmod(x, y); }
RT_SKY_MATH double m_asin(double x) { return ::asin(x); }
RT_SKY_MATH double m_tan(double x) { return ::tan(x); }

// comparison forms of max, min and clamp (NaN passes through as in <algorithm>)
template <class T>
RT_SKY_HD T mx(T a, T b) { return (a < b) ? b : a; }
template <class T>
RT_SKY_HD T mn(T a, T b) { return (b < a) ? b : a; }
template <class T>
RT_SKY_HD T cl(T v, T lo, T hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

struct V3 {
    double x, y, z;
};
RT_SKY_HD double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// ---- hashes (SphericalPartition, :308-340) ----
RT_SKY_HD uint64_t mix64(uint64_t h) {
    h ^= h >> 30;
    h *= 0xbf58476d1ce4e5b9ULL;
    h ^= h >> 27;
    h *= 0x94d049bb133111ebULL;
    h ^= h >> 31;
    return h;
}
RT_SKY_HD uint64_t hash_coords(uint32_t r, uint32_t s, uint64_t seed) {
    return mix64(seed ^ (static_cast<uint64_t>(r) * 0x9e3779b97f4a7c15ULL) ^ (static_cast<uint64_t>(s) * 0xbf58476d1ce4e5b9ULL));
}
RT_SKY_HD uint64_t hash_3d(int32_t x, int32_t y, int32_t z, uint64_t seed) {
    return mix64(seed ^ (static_cast<uint64_t>(static_cast<uint32_t>(x)) * 0x9e3779b97f4a7c15ULL) ^
                 (static_cast<uint64_t>(static_cast<uint32_t>(y)) * 0xbf58476d1ce4e5b9ULL) ^
                 (static_cast<uint64_t>(static_cast<uint32_t>(z)) * 0x94d049bb133111ebULL));
}
RT_SKY_HD double unit(uint64_t h) { return static_cast<double>(h & 0x001FFFFFFFFFFFFFULL) * (1.0 / 9007199254740992.0); }
RT_SKY_HD uint32_t sectors_of_ring(uint32_t ring, uint32_t rings) {
    const double zc = -1.0 + (2.0 * static_cast<double>(ring) + 1.0) / static_cast<double>(rings);
    const double st = sqrt(mx(1.0 - zc * zc, 1.0e-6));
    return static_cast<uint32_t>(mx(1.0, round(static_cast<double>(rings) * kPi * 0.5 * st)));
}

// A size or luminosity distribution (:342-385): 0 uniform, 1 power law, 2
// truncated exponential, 3 log-normal, 4 two-part; the terms that depend only
// on its parameters are formed once (make_dist), the rest per sample (draw).
struct Dist {
    uint32_t kind;
    double lo, hi, shape;
    double k0, k1, k2;
    bool log_uniform;  // power law of exponent 1
};
RT_SKY_HD Dist make_dist(uint32_t kind, double lo, double hi, double shape) {
    Dist d{kind, lo, hi, shape, 0.0, 0.0, 0.0, false};
    if (lo >= hi) return d;
    if (kind == 1u) {
        const double alpha = mx(shape, 0.05);
        if (fabs(alpha - 1.0) < 1.0e-4) {
            d.log_uniform = true;
            d.k0 = hi / lo;
        } else {
            const double e = 1.0 - alpha;
            d.k0 = m_pow(lo, e);
            d.k1 = m_pow(hi, e);
            d.k2 = 1.0 / e;
        }
    } else if (kind == 2u) {
        d.k0 = mx(shape, 0.1);                   // rate
        d.k1 = 1.0 - m_exp(-d.k0 * (hi - lo));   // normalisation
    } else if (kind == 3u) {
        const double a = m_log(mx(lo, 1.0e-12)), b = m_log(mx(hi, 1.0e-11));
        d.k0 = 0.5 * (a + b);
        d.k1 = cl(shape * 0.35, 0.05, 2.5) * (b - a);
    }
    return d;
}
// One sample from one hash.
RT_SKY_HD double draw(const Dist& d, uint64_t h) {
    const double u = unit(h);
    const double lo = d.lo, hi = d.hi;
    if (lo >= hi) return lo;
    switch (d.kind) {
        case 1:
            if (d.log_uniform) return lo * m_pow(d.k0, u);
            return cl(m_pow(mx((1.0 - u) * d.k0 + u * d.k1, 1.0e-30), d.k2), lo, hi);
        case 2:
            return lo - m_log(mx(1.0 - u * d.k1, 1.0e-15)) / d.k0;
        case 3: {
            const double u2 = mx(unit(h ^ 0x94d049bb133111ebULL), 1.0e-15);
            const double z = sqrt(-2.0 * m_log(mx(u, 1.0e-15))) * m_cos(2.0 * kPi * u2);
            return cl(m_exp(d.k0 + d.k1 * z), lo, hi);
        }
        case 4: {
            if (u < 0.85) return lo + (u / 0.85) * (lo + 0.12 * (hi - lo) - lo);
            const double split = lo + 0.60 * (hi - lo);
            return split + ((u - 0.85) / 0.15) * (hi - split);
        }
        default:
            return lo + u * (hi - lo);
    }
}
RT_SKY_HD double draw(uint32_t kind, double lo, double hi, double shape, uint64_t h) {
    return draw(make_dist(kind, lo, hi, shape), h);
}

// ---- value noise (:387-448) ----
RT_SKY_HD float lattice(int32_t x, int32_t y, int32_t z) {
    // the reference's 32-bit integer hash, in unsigned (wrapping) arithmetic
    uint32_t n = static_cast<uint32_t>(x) + static_cast<uint32_t>(y) * 57u + static_cast<uint32_t>(z) * 113u;
    n = (n << 13) ^ n;
    const uint32_t v = (n * (n * n * 15731u + 789221u) + 1376312589u) & 0x7fffffffu;
    return 1.0f - static_cast<float>(v) * (1.0f / 1073741824.0f);
}
RT_SKY_HD float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
RT_SKY_HD float vnoise(float x, float y, float z) {
    const int32_t xi = static_cast<int32_t>(floorf(x)), yi = static_cast<int32_t>(floorf(y)),
                  zi = static_cast<int32_t>(floorf(z));
    const float u = fade(x - static_cast<float>(xi)), v = fade(y - static_cast<float>(yi)),
                w = fade(z - static_cast<float>(zi));
    const float c00 = lattice(xi, yi, zi) * (1.0f - u) + lattice(xi + 1, yi, zi) * u;
    const float c10 = lattice(xi, yi + 1, zi) * (1.0f - u) + lattice(xi + 1, yi + 1, zi) * u;
    const float c01 = lattice(xi, yi, zi + 1) * (1.0f - u) + lattice(xi + 1, yi, zi + 1) * u;
    const float c11 = lattice(xi, yi + 1, zi + 1) * (1.0f - u) + lattice(xi + 1, yi + 1, zi + 1) * u;
    const float c0 = c00 * (1.0f - v) + c10 * v;
    const float c1 = c01 * (1.0f - v) + c11 * v;
    return c0 * (1.0f - w) + c1 * w;
}
RT_SKY_HD float fbm(float x, float y, float z, int octaves, float rough) {
    float total = 0.0f, amp = 1.0f, freq = 1.0f, norm = 0.0f;
    #pragma unroll 1
    for (int i = 0; i < octaves; ++i) {
        total += vnoise(x * freq, y * freq, z * freq) * amp;
        norm += amp;
        amp *= rough;
        freq *= 2.02f;
    }
    return total / mx(norm, 1e-5f);
}
RT_SKY_HD float ridged(float x, float y, float z, int octaves, float rough) {
    float total = 0.0f, amp = 1.0f, freq = 1.0f, norm = 0.0f;
    #pragma unroll 1
    for (int i = 0; i < octaves; ++i) {
        float v = 1.0f - fabsf(vnoise(x * freq, y * freq, z * freq));
        v *= v;
        total += v * amp;
        norm += amp;
        amp *= rough;
        freq *= 2.05f;
    }
    return total / mx(norm, 1e-5f);
}

// Yaw about z, pitch about y, roll about x, in degrees (:450-477).
RT_SKY_HD V3 rotate(const V3& v, double yaw, double pitch, double roll) {
    const double cy = m_cos(yaw * kDegToRad), sy = m_sin(yaw * kDegToRad);
    const double cp = m_cos(pitch * kDegToRad), sp = m_sin(pitch * kDegToRad);
    const double cr = m_cos(roll * kDegToRad), sr = m_sin(roll * kDegToRad);
    const double x1 = v.x * cy - v.y * sy, y1 = v.x * sy + v.y * cy, z1 = v.z;
    const double x2 = x1 * cp + z1 * sp, y2 = y1, z2 = -x1 * sp + z1 * cp;
    return {x2, y2 * cr - z2 * sr, y2 * sr + z2 * cr};
}

// HSV hue shift and saturation scale of a float colour (:480-526).
RT_SKY_HD void hue_saturation(float* rgb, double hue_rad, double sat) {
    if (hue_rad == 0.0 && sat == 1.0) return;
    const float r = rgb[0], g = rgb[1], b = rgb[2];
    const float hi = mx(mx(r, g), b), lo = mn(mn(r, g), b), delta = hi - lo;
    float h = 0.0f;
    if (delta > 1e-8f) {
        if (hi == r) h = fmodf((g - b) / delta, 6.0f);
        else if (hi == g) h = (b - r) / delta + 2.0f;
        else h = (r - g) / delta + 4.0f;
        h *= 60.0f;
        if (h < 0.0f) h += 360.0f;
    }
    const float s0 = (hi > 1e-8f) ? (delta / hi) : 0.0f;
    h += static_cast<float>(hue_rad * (180.0 / kPi));
    h = fmodf(h, 360.0f);
    if (h < 0.0f) h += 360.0f;
    const float s1 = cl(s0 * static_cast<float>(sat), 0.0f, 1.0f);
    const float c = hi * s1;
    const float x = c * (1.0f - fabsf(fmodf(h / 60.0f, 2.0f) - 1.0f));
    const float m = hi - c;
    float r2, g2, b2;
    if (h < 60.0f) { r2 = c; g2 = x; b2 = 0.0f; }
    else if (h < 120.0f) { r2 = x; g2 = c; b2 = 0.0f; }
    else if (h < 180.0f) { r2 = 0.0f; g2 = c; b2 = x; }
    else if (h < 240.0f) { r2 = 0.0f; g2 = x; b2 = c; }
    else if (h < 300.0f) { r2 = x; g2 = 0.0f; b2 = c; }
    else { r2 = c; g2 = 0.0f; b2 = x; }
    rgb[0] = r2 + m;
    rgb[1] = g2 + m;
    rgb[2] = b2 + m;
}

// A unit vector from three floats of the profile, or the fallback.
RT_SKY_HD V3 unit_or(const float* v, V3 fallback) {
    const double a = static_cast<double>(v[0]), b = static_cast<double>(v[1]), c = static_cast<double>(v[2]);
    const double len = sqrt(a * a + b * b + c * c);
    return (len > 1e-9) ? V3{a / len, b / len, c / len} : fallback;
}

// An orthonormal pair perpendicular to a unit direction, as the layers build it.
RT_SKY_HD void tangents(const V3& d, V3& u1, V3& u2) {
    u1 = (fabs(d.z) < 0.9) ? V3{-d.y, d.x, 0.0} : V3{0.0, -d.z, d.y};
    const double len = sqrt(u1.x * u1.x + u1.y * u1.y + u1.z * u1.z);
    u1.x /= len;
    u1.y /= len;
    u1.z /= len;
    u2 = {d.y * u1.z - d.z * u1.y, d.z * u1.x - d.x * u1.z, d.x * u1.y - d.y * u1.x};
}

// Point of a hashed cell of the 3-D direction grid (cell corner + hashed offset), normalised.
RT_SKY_HD bool cell_point(int32_t ix, int32_t iy, int32_t iz, uint64_t h, V3& out) {
    const double ox = static_cast<double>(ix) + unit(h + 11ULL);
    const double oy = static_cast<double>(iy) + unit(h + 23ULL);
    const double oz = static_cast<double>(iz) + unit(h + 37ULL);
    const double len = sqrt(ox * ox + oy * oy + oz * oz);
    if (len <= 1.0e-9) return false;
    out = {ox / len, oy / len, oz / len};
    return true;
}

// ---- point-spread functions of stars (:671-746) ----
RT_SKY_HD double bessel_j1(double x) {
    // polynomial approximations of J1 (Abramowitz & Stegun 9.4.4 and 9.4.6)
    const double ax = fabs(x);
    if (ax < 3.75) {
        const double y = (x / 3.75) * (x / 3.75);
        return x * (0.5 + y * (-0.56249985 + y * (0.21093573 + y * (-0.03954289 + y * (0.00443319 - y * 0.00031761)))));
    }
    const double y = 3.75 / ax;
    const double f0 = 0.79788456 + y * (-0.00000077 + y * (-0.00552740 + y * (0.00009512 + y * (0.00137237 - y * 0.00072805))));
    const double t0 = ax - 2.35619449 + y * (0.04411179 + y * (-0.00008449 + y * (-0.00076126 + y * (0.00009185 + y * 0.00008544))));
    const double v = (f0 / sqrt(ax)) * m_cos(t0);
    return (x < 0.0) ? -v : v;
}

RT_SKY_HD double star_psf(double theta_sq, double sigma, double eff_sq, double pix, const SkyProfile& s, double lx,
                          double ly, uint32_t model) {
    const double theta = sqrt(mx(theta_sq, 0.0));
    switch (model) {
        case 6: {  // pinpoint
            const double tight = cl(s.star_dirac_concentration, 0.1, 0.999);
            const double w = mx(pix * (1.0 - tight) * 0.4, 1.0e-9);
            return m_exp(-theta_sq / (2.0 * w * w));
        }
        case 7: {  // cinematic bloom
            const double core = m_exp(-theta_sq / (2.0 * eff_sq));
            const double w = mx(sigma * cl(s.star_bloom_radius, 1.0, 30.0), pix * 3.5);
            return core + s.star_bloom_intensity * 1.8 * m_exp(-theta / w);
        }
        case 1: {  // Lorentzian
            const double g2 = eff_sq * mx(s.star_profile_param, 0.05);
            return (g2 / (g2 + theta_sq)) + 0.25 * (g2 / (g2 + theta_sq * 0.25));
        }
        case 2: {  // Moffat
            const double beta = cl(s.star_profile_param, 1.05, 8.0);
            const double scale = mx(eff_sq * s.star_profile_param2, 1.0e-12);
            return m_pow(1.0 + theta_sq / scale, -beta);
        }
        case 3: {  // Airy
            const double v = kPi * theta / mx(sigma, 1.0e-8);
            if (v < 1.0e-4) return 1.0;
            const double j = bessel_j1(v);
            const double core = (2.0 * j / v) * (2.0 * j / v);
            return mn(core * mx(s.star_profile_param2, 0.1), 2.0);
        }
        case 4: {  // hard disc
            const double rad = mx(sigma, pix * 0.5);
            const double soft = cl(s.star_profile_softness, 0.001, 1.0);
            const double edge = mx(pix * 0.4, rad * soft);
            return 1.0 - cl((theta - (rad - edge)) / mx(2.0 * edge, 1.0e-9), 0.0, 1.0);
        }
        case 5: {  // diffraction spikes
            const double core = m_exp(-theta_sq / (2.0 * eff_sq));
            const double ang = m_atan2(ly, lx) + s.star_spike_angle_deg * (kPi / 180.0);
            const double ns = (s.star_spike_count == 6u) ? 3.0 : ((s.star_spike_count == 8u) ? 4.0 : 2.0);
            const double beam = m_pow(fabs(m_cos(ns * ang)), 32.0);
            const double len = mx(sigma * cl(s.star_spike_length, 0.5, 60.0), pix * 8.0);
            return core + s.star_spike_intensity * 2.5 * beam * m_exp(-theta / len);
        }
        default:  // Gaussian with a faint exponential wing
            return m_exp(-theta_sq / (2.0 * eff_sq)) + 0.06 * m_exp(-theta / (4.0 * mx(sigma, 1.0e-8)));
    }
}

RT_SKY_HD void star_tint(double t, double variation, float* out) {
    float r = 1.0f, g = 1.0f, b = 1.0f;
    if (t < 0.20) { r = 1.55f; g = 0.65f; b = 0.35f; }
    else if (t < 0.45) { r = 1.35f; g = 1.05f; b = 0.70f; }
    else if (t < 0.70) { r = 1.05f; g = 1.05f; b = 1.05f; }
    else if (t < 0.88) { r = 0.80f; g = 0.95f; b = 1.35f; }
    else { r = 0.65f; g = 0.80f; b = 1.60f; }
    const float m = static_cast<float>(cl(variation, 0.0, 3.0));
    out[0] = mx(0.0f, 1.0f + (r - 1.0f) * m);
    out[1] = mx(0.0f, 1.0f + (g - 1.0f) * m);
    out[2] = mx(0.0f, 1.0f + (b - 1.0f) * m);
}

// ---- layers ----

// Stars on a hashed 3-D grid around the direction (:769-913).
RT_SKY_HD_NOINLINE void stars(const V3& dir, const SkyProfile& s, double fov, double time, double* acc) {
    if (!s.stars_enabled || s.star_density <= 0.0) return;
    const uint64_t seed = static_cast<uint64_t>(s.seed);
    const double q = mx(s.quality_factor * s.star_quality_factor, 0.05);
    const double dens = cl(s.star_density * q, 0.01, 100.0);
    const double res = cl(14.0 * sqrt(dens), 6.0, 120.0);
    const double pix = mx(fov / 1080.0, 1.0e-7);
    const uint32_t model = s.star_profile_model;
    const V3 plane = unit_or(s.nebula_plane_normal, V3{0.0, 0.4472135955, 0.894427191});
    const int32_t cx = static_cast<int32_t>(floor(dir.x * res)), cy = static_cast<int32_t>(floor(dir.y * res)),
                  cz = static_cast<int32_t>(floor(dir.z * res));
    const double presence = cl(1.0 - (s.star_density * q) * 0.16, 0.01, 0.99);
    const Dist size_dist = make_dist(s.star_size_distribution, s.star_size_min, s.star_size_max, s.star_size_param);
    const Dist lum_dist = make_dist(s.star_luminosity_distribution, 0.2, 25.0, s.star_luminosity_param);
    const double size_scale = mx(s.star_size_scale, 0.05);
    #pragma unroll 1
    for (int32_t dz = -1; dz <= 1; ++dz)
        #pragma unroll 1
        for (int32_t dy = -1; dy <= 1; ++dy)
            #pragma unroll 1
            for (int32_t dx = -1; dx <= 1; ++dx) {
                const int32_t ix = cx + dx, iy = cy + dy, iz = cz + dz;
                const uint64_t h = hash_3d(ix, iy, iz, seed);
                if (unit(h) <= presence) continue;
                V3 sd;
                if (!cell_point(ix, iy, iz, h, sd)) continue;
                // the star's angular distance, size and support (the tests of its
                // distance and of the placement model are pure: a star that does not
                // move is measured first, so that most stars skip the placement model)
                double th2 = 0.0, rad = 0.0, sig = 0.0, sig2 = 0.0, support2 = 0.0;
                auto within = [&]() -> bool {
                    const double mu = dot(dir, sd);
                    if (mu <= 0.994) return false;
                    th2 = 2.0 * mx(0.0, 1.0 - mu);
                    rad = draw(size_dist, h + 31ULL) * size_scale;
                    const double sub = (model == 6u) ? 0.04 : 0.35;
                    sig = sqrt(rad * rad * (model == 4u ? 1.0 : 1.96) + pix * pix * sub);
                    sig2 = sig * sig;
                    double support = sig * 6.0;
                    if (model == 5u) support = mx(support, sig * cl(s.star_spike_length, 1.0, 60.0));
                    else if (model == 7u) support = mx(support, sig * cl(s.star_bloom_radius, 1.0, 30.0));
                    else if (model == 3u) support = mx(support, sig * 12.0);
                    else if (model == 1u || model == 2u) support = mx(support, sig * 10.0);
                    support2 = support * support;
                    return !(th2 > support2);
                };
                if (!s.dynamic_motion && !within()) continue;
                // placement models: 1 galactic disk, 2 fractal clusters, 3 two
                // populations, 4 spiral-arm density, 5 constellation associations
                if (s.star_placement_model == 1u) {
                    const double hp = dot(sd, plane);
                    const double p = m_exp(-fabs(hp) * cl(s.star_galactic_concentration, 0.2, 20.0));
                    if (unit(h + 101ULL) > (p * 0.95 + 0.05)) continue;
                } else if (s.star_placement_model == 2u) {
                    const float n = fbm(static_cast<float>(sd.x * 3.8), static_cast<float>(sd.y * 3.8),
                                        static_cast<float>(sd.z * 3.8), 3, 0.65f);
                    const double p = m_pow(cl((static_cast<double>(n) + 0.6) * 0.85, 0.0, 1.0), 3.0);
                    if (unit(h + 102ULL) > p) continue;
                } else if (s.star_placement_model == 3u) {
                    const double hp = dot(sd, plane);
                    if (unit(h + 103ULL) > 0.30) {
                        const double p = m_exp(-fabs(hp) * cl(s.star_galactic_concentration, 0.5, 15.0));
                        if (unit(h + 107ULL) > p) continue;
                    }
                } else if (s.star_placement_model == 4u) {
                    const double hp = dot(sd, plane);
                    const double phi = m_atan2(sd.y, sd.x);
                    const double arm = m_sin(2.0 * phi - 4.5 * m_log(mx(fabs(hp) + 0.2, 0.05)));
                    const double p = cl(m_exp(-fabs(hp) * 3.0) * (0.15 + 0.85 * (arm * 0.5 + 0.5)), 0.02, 1.0);
                    if (unit(h + 109ULL) > p) continue;
                } else if (s.star_placement_model == 5u) {
                    const float a = lattice(static_cast<int32_t>(sd.x * 5.0), static_cast<int32_t>(sd.y * 5.0),
                                            static_cast<int32_t>(sd.z * 5.0));
                    if (unit(h + 111ULL) > (static_cast<double>(fabsf(a)) * 0.9 + 0.1)) continue;
                }
                if (s.dynamic_motion) {
                    const double rate = s.motion_speed * 0.012;
                    const double phase = unit(h + 47ULL) * kTwoPi;
                    const double ang = m_sin(time * 0.18 + phase) * rate;
                    sd = rotate(sd, ang * (180.0 / kPi), 0.0, 0.0);
                    if (!within()) continue;
                }
                const double wu = cl(th2 / support2, 0.0, 1.0);
                const double window = (1.0 - wu) * (1.0 - wu);
                double lum = draw(lum_dist, h + 53ULL) * s.star_brightness;
                if (s.dynamic_motion && s.star_scintillation > 0.0) {
                    const double tw = unit(h + 67ULL) * kTwoPi;
                    lum *= (1.0 + s.star_scintillation * m_sin(time * 3.8 + tw));
                }
                V3 u1, u2;
                tangents(sd, u1, u2);
                const V3 d{dir.x - sd.x, dir.y - sd.y, dir.z - sd.z};
                const double psf = star_psf(th2, sig, sig2, pix, s, dot(d, u1), dot(d, u2), model);
                const double ratio = cl((rad * rad) / sig2, 0.02, 4.0);
                const double flux = lum * ratio * psf * window;
                float tint[3];
                star_tint(cl(unit(h + 79ULL) + s.star_temperature_bias * 0.4, 0.0, 1.0), s.star_color_variation, tint);
                acc[0] += flux * static_cast<double>(tint[0]);
                acc[1] += flux * static_cast<double>(tint[1]);
                acc[2] += flux * static_cast<double>(tint[2]);
            }
}

// Emission nebulae along the galactic plane (:915-1008).
RT_SKY_HD_NOINLINE void nebulae(const V3& dir, const SkyProfile& s, double zoom, double* acc) {
    if (!s.nebula_enabled || s.nebula_intensity <= 0.0) return;
    const V3 plane = unit_or(s.nebula_plane_normal, V3{0.0, 0.4472135955, 0.894427191});
    const double hgt = dot(dir, plane);
    const double thick = mx(s.nebula_plane_thickness, 0.02);
    const double fall = cl(s.nebula_plane_falloff, 1.0, 6.0);
    const double disc = m_exp(-m_pow(fabs(hgt) / thick, fall));
    const V3 asym = unit_or(s.nebula_asymmetry_dir, V3{0.7071067812, 0.0, 0.7071067812});
    const double cpsi = dot(dir, asym);
    const double asym_env = m_pow(cl((1.0 + cpsi) * 0.5, 0.0, 1.0), cl(s.nebula_asymmetry * 2.5 + 0.1, 0.1, 8.0));
    const double glow = s.nebula_core_glow * m_exp(-2.5 * mx(0.0, 1.0 - cpsi));
    const double q = mx(s.quality_factor * s.nebula_quality_factor, 0.05);
    int oct = cl(static_cast<int>(static_cast<double>(s.nebula_octaves) * sqrt(q)), 1, 8);
    if (s.adaptive_fov_quality && zoom > 1.2) oct = mn(8, oct + static_cast<int>(floor(log2(zoom))));
    const float freq = static_cast<float>(s.nebula_frequency);
    const float rough = static_cast<float>(cl(s.nebula_roughness, 0.1, 0.95));
    const float sf = static_cast<float>(s.seed % 1024u) * 1.37f;
    float dx = static_cast<float>(dir.x), dy = static_cast<float>(dir.y), dz = static_cast<float>(dir.z);
    if (s.nebula_curl_strength > 0.01) {
        const float k = static_cast<float>(s.nebula_curl_strength * 0.25);
        const float cx = vnoise(dy * 2.0f, dz * 2.0f, sf);
        const float cy = vnoise(dz * 2.0f, dx * 2.0f, sf + 7.1f);
        const float cz = vnoise(dx * 2.0f, dy * 2.0f, sf + 13.3f);
        dx += cx * k;
        dy += cy * k;
        dz += cz * k;
        const float inv = 1.0f / mx(sqrtf(dx * dx + dy * dy + dz * dz), 1.0e-6f);
        dx *= inv;
        dy *= inv;
        dz *= inv;
    }
    const uint32_t layers = cl(static_cast<uint32_t>(static_cast<double>(s.nebula_layer_count) * q + 0.4), 1u, 5u);
    double er = 0.0, eg = 0.0, eb = 0.0;
    const float sep = static_cast<float>(cl(s.nebula_color_separation, 0.5, 3.0));
    const float gas = static_cast<float>(cl(s.nebula_gas_contrast, 0.5, 3.0));
    const float ion = static_cast<float>(cl(s.nebula_ionization_glow, 0.0, 3.0));
    const float* c1 = s.nebula_emission_color;
    const float* c2 = s.nebula_secondary_color;
    const float* c3 = s.nebula_tertiary_color;
    #pragma unroll 1
    for (uint32_t L = 0; L < layers; ++L) {
        const float off = static_cast<float>(L) * 17.3f * static_cast<float>(s.nebula_layer_spread);
        const float sc = 1.0f + static_cast<float>(L) * 0.75f * static_cast<float>(s.nebula_layer_spread);
        const float n1 = fbm(dx * freq * sc + sf + off, dy * freq * sc - sf * 0.7f, dz * freq * sc + 13.5f + off, oct, rough);
        const float e1 = powf(mx(0.0f, (n1 + 0.18f) * 1.05f), 1.8f * gas);
        const float n2 = fbm(dx * freq * 1.85f * sc - 27.1f + off * sep, dy * freq * 1.85f * sc + sf * 0.5f,
                             dz * freq * 1.85f * sc - 11.2f, oct, rough);
        const float e2 = powf(mx(0.0f, (n2 + 0.12f) * 1.10f), 2.2f * gas) * ion;
        const float n3 = fbm(dx * freq * 2.7f * sc + 43.0f, dy * freq * 2.7f * sc + off * (sep * 1.3f),
                             dz * freq * 2.7f * sc - sf, oct, rough);
        const float e3 = powf(mx(0.0f, (n3 + 0.05f) * 0.95f), 2.4f * gas);
        const double w = 1.0 / (1.0 + 0.45 * static_cast<double>(L));
        er += (static_cast<double>(e1 * c1[0]) + static_cast<double>(e2 * c2[0] * 0.35f) + static_cast<double>(e3 * c3[0])) * w;
        eg += (static_cast<double>(e1 * c1[1] * 0.30f) + static_cast<double>(e2 * c2[1]) +
               static_cast<double>(e3 * c3[1] * 0.75f)) * w;
        eb += (static_cast<double>(e1 * c1[2] * 0.65f) + static_cast<double>(e2 * c2[2] * 0.95f) +
               static_cast<double>(e3 * c3[2] * 0.20f)) * w;
    }
    const float nd = ridged(dx * freq * 2.6f + 71.3f, dy * freq * 2.6f - 39.4f, dz * freq * 2.6f + sf, oct, 0.6f);
    const float tau = mx(0.0f, nd - 0.26f) * static_cast<float>(s.nebula_absorption_density * 2.6);
    const double ext = m_exp(-static_cast<double>(tau));
    const double env = (disc * asym_env + glow) * ext * (s.nebula_intensity * s.nebula_quality_factor);
    acc[0] += er * env;
    acc[1] += eg * env;
    acc[2] += eb * env;
}

// Cell of the equal-area ring/sector partition and its jittered centre (galaxies, clusters).
RT_SKY_HD V3 ring_cell_centre(uint32_t r, uint32_t s, uint32_t rings, uint32_t sectors, uint64_t h, uint64_t kz,
                              uint64_t kp) {
    const double zc = -1.0 + (2.0 * static_cast<double>(r) + 1.0) / static_cast<double>(rings);
    const double pc = kTwoPi * (static_cast<double>(s) + 0.5) / static_cast<double>(sectors);
    const double z = cl(zc + (unit(h + kz) - 0.5) * (1.6 / static_cast<double>(rings)), -1.0, 1.0);
    const double p = m_remainder(pc + (unit(h + kp) - 0.5) * (1.6 * kTwoPi / static_cast<double>(sectors)), kTwoPi);
    const double rxy = sqrt(mx(1.0 - z * z, 0.0));
    return {rxy * m_cos(p), rxy * m_sin(p), z};
}

// Galaxies (:1010-1174).
RT_SKY_HD_NOINLINE void galaxies(const V3& dir, const SkyProfile& s, double* acc) {
    if (!s.galaxies_enabled || s.galaxy_density <= 0.0) return;
    const uint64_t seed = static_cast<uint64_t>(s.seed) ^ 0x6a09e667f3bcc908ULL;
    const uint32_t rings = static_cast<uint32_t>(cl(round(14.0 * sqrt(s.galaxy_density)), 4.0, 36.0));
    const uint32_t rc = cl(static_cast<uint32_t>((cl(dir.z, -1.0, 1.0) + 1.0) * 0.5 * static_cast<double>(rings)), 0u,
                           rings - 1u);
    double pd = m_atan2(dir.y, dir.x);
    if (pd < 0.0) pd += kTwoPi;
    const double presence = cl(1.0 - s.galaxy_density * 0.25, 0.02, 0.99);
    #pragma unroll 1
    for (int dr = -1; dr <= 1; ++dr) {
        const int rcand = static_cast<int>(rc) + dr;
        if (rcand < 0 || rcand >= static_cast<int>(rings)) continue;
        const uint32_t ri = static_cast<uint32_t>(rcand);
        const uint32_t ns = sectors_of_ring(ri, rings);
        const uint32_t sc = cl(static_cast<uint32_t>(pd / kTwoPi * static_cast<double>(ns)), 0u, ns - 1u);
        #pragma unroll 1
        for (int ds = -1; ds <= 1; ++ds) {
            const uint32_t si = (sc + ns + ds) % ns;
            const uint64_t h = hash_coords(ri, si, seed);
            if (unit(h) > presence) continue;
            const V3 g = ring_cell_centre(ri, si, rings, ns, h, 3ULL, 7ULL);
            const double mu = dot(dir, g);
            if (mu <= 0.9985) continue;
            const double sep2 = 2.0 * mx(0.0, 1.0 - mu);
            const double size = draw(s.galaxy_size_distribution, s.galaxy_size_min, s.galaxy_size_max,
                                     s.galaxy_size_param, h + 13ULL) * s.galaxy_size_scale;
            if (sep2 > 9.0 * size * size) continue;
            V3 t1, t2;
            tangents(g, t1, t2);
            const double pa = unit(h + 17ULL) * kTwoPi;
            const double cpa = m_cos(pa), spa = m_sin(pa);
            const V3 u1{t1.x * cpa + t2.x * spa, t1.y * cpa + t2.y * spa, t1.z * cpa + t2.z * spa};
            const V3 u2{-t1.x * spa + t2.x * cpa, -t1.y * spa + t2.y * cpa, -t1.z * spa + t2.z * cpa};
            const double cinc = cl(1.0 - unit(h + 23ULL) * s.galaxy_inclination_variance, 0.12, 1.0);
            const double sinc = sqrt(mx(1.0 - cinc * cinc, 0.0));
            const V3 d{dir.x - g.x, dir.y - g.y, dir.z - g.z};
            const double xo = dot(d, u1) / mx(size, 1.0e-6);
            const double yo = dot(d, u2) / mx(size, 1.0e-6);
            const double xd = xo, yd = yo / cinc;
            const double rd = sqrt(xd * xd + yd * yd);
            const double phd = m_atan2(yd, xd);
            uint32_t morph = s.galaxy_morphology_model;
            if (morph == 0u) {
                const double w1 = mx(s.galaxy_weight_grand_design, 0.0), w2 = mx(s.galaxy_weight_flocculent, 0.0),
                             w3 = mx(s.galaxy_weight_barred, 0.0), w4 = mx(s.galaxy_weight_elliptical, 0.0),
                             w5 = mx(s.galaxy_weight_lenticular, 0.0), w6 = mx(s.galaxy_weight_ring, 0.0);
                double sum = w1 + w2 + w3 + w4 + w5 + w6;
                if (sum <= 1.0e-9) sum = 1.0;
                const double pick = unit(h + 999ULL) * sum;
                if (pick < w1) morph = 1u;
                else if (pick < w1 + w2) morph = 2u;
                else if (pick < w1 + w2 + w3) morph = 3u;
                else if (pick < w1 + w2 + w3 + w4) morph = 4u;
                else if (pick < w1 + w2 + w3 + w4 + w5) morph = 5u;
                else morph = 6u;
            }
            double core, disk = 0.0;
            double tc[3] = {1.25, 1.05, 0.70}, td[3] = {0.65, 0.85, 1.35};
            if (morph == 4u) {  // elliptical: Sersic bulge
                const double b = 2.0 * s.galaxy_bulge_sersic_index - 0.333333;
                core = m_exp(-cl(b * m_pow(rd, 1.0 / s.galaxy_bulge_sersic_index), 0.0, 30.0));
                tc[0] = 1.35; tc[1] = 1.00; tc[2] = 0.65;
            } else if (morph == 5u) {  // lenticular with a dust ring
                core = m_exp(-rd * 3.5);
                disk = m_exp(-rd * 1.8);
                const double rdist = fabs(rd - 0.65);
                disk *= (1.0 - (1.0 - m_exp(-rdist * rdist / 0.008)) * s.galaxy_dust_lane_opacity);
                tc[0] = 1.20; tc[1] = 1.05; tc[2] = 0.80;
                td[0] = 0.95; td[1] = 0.95; td[2] = 0.90;
            } else if (morph == 3u) {  // barred spiral
                core = m_exp(-rd * rd * 6.0);
                const double bl = 0.55 * cl(s.galaxy_bar_strength, 0.1, 2.0), bw = 0.15;
                const double bar = m_exp(-(xd * xd) / (2.0 * bl * bl) - (yd * yd) / (2.0 * bw * bw));
                const double arms = 0.5 + 0.5 * m_cos(2.0 * (phd - rd * 3.5 * s.galaxy_pitch_angle));
                disk = (bar * 0.7 + m_exp(-rd * 2.2) * arms * 0.5);
            } else if (morph == 2u) {  // flocculent
                core = m_exp(-rd * 4.0);
                const float cn = fbm(static_cast<float>(xd * 6.0), static_cast<float>(yd * 6.0), static_cast<float>(h & 0xFFu),
                                     3, 0.6f);
                const double arms = 0.5 + 0.5 * m_cos(6.0 * phd - rd * 7.0 * s.galaxy_pitch_angle + static_cast<double>(cn) * 2.5);
                disk = m_exp(-rd * 2.5) * arms * (1.0 + s.galaxy_clumpiness * static_cast<double>(cn));
            } else if (morph == 6u) {  // ring
                core = m_exp(-rd * rd * 8.0) * 1.2;
                const double diff = fabs(rd - 0.70);
                disk = m_exp(-(diff * diff) / (2.0 * 0.12 * 0.12)) * 1.4;
                td[0] = 0.45; td[1] = 0.80; td[2] = 1.65;
            } else {  // grand-design spiral
                core = m_exp(-rd * rd * 4.0);
                const double arms = 0.5 + 0.5 * m_cos(s.galaxy_spiral_arms * phd - rd * 4.8 * s.galaxy_pitch_angle);
                disk = m_exp(-rd * 2.2) * arms;
            }
            if (morph != 4u && s.galaxy_dust_lane_opacity > 0.0) {
                const double near = yo * sinc;
                if (near > 0.0) {
                    const double lane = m_exp(-fabs(near - 0.18) * 9.0) * s.galaxy_dust_lane_opacity;
                    core *= (1.0 - lane * 0.85);
                    disk *= (1.0 - lane * 0.65);
                }
            }
            const double cr = cl(s.galaxy_core_ratio, 0.0, 1.0);
            const double f = (core * cr + disk * (1.0 - cr)) * s.galaxy_brightness * 1.6;
            const double tm = 0.8 + 0.4 * unit(h + 29ULL);
            acc[0] += f * (cr * tc[0] + (1.0 - cr) * td[0]) * tm;
            acc[1] += f * (cr * tc[1] + (1.0 - cr) * td[1]);
            acc[2] += f * (cr * tc[2] + (1.0 - cr) * td[2]) * (2.0 - tm);
        }
    }
}

// Star clusters: Plummer halo and resolved members (:1176-1318).
RT_SKY_HD_NOINLINE void clusters(const V3& dir, const SkyProfile& s, double fov, double* acc) {
    if (!s.clusters_enabled || s.cluster_density <= 0.0) return;
    const uint64_t seed = static_cast<uint64_t>(s.seed) ^ 0xbb67ae8584caa73bULL;
    const double dens = mx(s.cluster_density, 0.01);
    const uint32_t rings = static_cast<uint32_t>(cl(round(10.0 * sqrt(dens)), 3.0, 36.0));
    const uint32_t rc = cl(static_cast<uint32_t>((cl(dir.z, -1.0, 1.0) + 1.0) * 0.5 * static_cast<double>(rings)), 0u,
                           rings - 1u);
    double pd = m_atan2(dir.y, dir.x);
    if (pd < 0.0) pd += kTwoPi;
    const double presence = cl(1.0 - dens * 0.16, 0.01, 0.99);
    const V3 plane = unit_or(s.nebula_plane_normal, V3{0.0, 0.4472135955, 0.894427191});
    const V3 asym = unit_or(s.nebula_asymmetry_dir, V3{0.7071067812, 0.0, 0.7071067812});
    const double pix = fov / 1080.0;
    const uint32_t mprof = s.cluster_inherit_star_profile ? s.star_profile_model : s.cluster_star_profile_model;
    #pragma unroll 1
    for (int dr = -1; dr <= 1; ++dr) {
        const int rcand = static_cast<int>(rc) + dr;
        if (rcand < 0 || rcand >= static_cast<int>(rings)) continue;
        const uint32_t ri = static_cast<uint32_t>(rcand);
        const uint32_t ns = sectors_of_ring(ri, rings);
        const uint32_t sc = cl(static_cast<uint32_t>(pd / kTwoPi * static_cast<double>(ns)), 0u, ns - 1u);
        #pragma unroll 1
        for (int ds = -1; ds <= 1; ++ds) {
            const uint32_t si = (sc + ns + ds) % ns;
            const uint64_t h = hash_coords(ri, si, seed);
            if (unit(h) > presence) continue;
            const V3 c = ring_cell_centre(ri, si, rings, ns, h, 5ULL, 9ULL);
            if (s.cluster_placement_model == 0u) {  // globular halo around the asymmetry direction
                const double cg = dot(c, asym);
                const double p = 1.0 / (1.0 + (1.0 - cg) / mx(s.cluster_halo_radius * s.cluster_halo_radius, 0.04));
                if (unit(h + 99ULL) > p) continue;
            } else if (s.cluster_placement_model == 1u) {  // open clusters near the plane
                const double hc = dot(c, plane);
                const double p = m_exp(-(hc * hc) / mx(s.cluster_plane_scale_height * s.cluster_plane_scale_height, 0.005));
                if (unit(h + 99ULL) > p) continue;
            }
            const double mu = dot(dir, c);
            if (mu <= 0.9985) continue;
            const double sep2 = 2.0 * mx(0.0, 1.0 - mu);
            const double crad = draw(s.cluster_size_distribution, s.cluster_size_min, s.cluster_size_max, 1.5, h + 17ULL) *
                                s.cluster_size_scale;
            const double r2 = crad * crad;
            if (sep2 > 9.0 * r2) continue;
            if (s.cluster_halo_intensity > 0.0) {
                const double cd = r2 * 0.40 * mx(s.cluster_spread_factor, 0.1);
                const double plummer = 1.0 / m_pow(1.0 + sep2 / mx(cd, 1.0e-7), s.cluster_concentration);
                const double f = plummer * s.cluster_brightness * cl(s.cluster_halo_intensity, 0.0, 2.0) * 0.75;
                acc[0] += f * static_cast<double>(s.cluster_core_tint[0]);
                acc[1] += f * static_cast<double>(s.cluster_core_tint[1]);
                acc[2] += f * static_cast<double>(s.cluster_core_tint[2]);
            }
            if (s.cluster_stars_enabled && s.cluster_member_count > 0u) {
                V3 u1, u2;
                tangents(c, u1, u2);
                const uint32_t members =
                    cl(static_cast<uint32_t>(static_cast<double>(s.cluster_member_count) * s.cluster_quality_factor), 4u, 256u);
                const double rcore = crad * 0.50 * mx(s.cluster_spread_factor, 0.1);
                #pragma unroll 1
                for (uint32_t m = 0; m < members; ++m) {
                    const uint64_t mh = hash_coords(ri * 1000u + si, m, seed ^ 0x3c6ef372fe94f82bULL);
                    const double ur = cl(unit(mh), 0.001, 0.96);
                    const double p23 = m_pow(ur, 2.0 / 3.0);
                    const double rm = rcore * sqrt(p23 / mx(1.0 - m_pow(ur, 2.0 / 3.0), 1.0e-4));
                    const double pm = kTwoPi * unit(mh + 13ULL);
                    const double dxm = rm * m_cos(pm), dym = rm * m_sin(pm);
                    const double px = c.x + u1.x * dxm + u2.x * dym, py = c.y + u1.y * dxm + u2.y * dym,
                                 pz = c.z + u1.z * dxm + u2.z * dym;
                    const double ml = sqrt(px * px + py * py + pz * pz);
                    const V3 md{px / ml, py / ml, pz / ml};
                    const double mum = dot(dir, md);
                    if (mum <= 0.9994) continue;
                    const double th2 = 2.0 * mx(0.0, 1.0 - mum);
                    const double mrad = mx(s.cluster_member_size, 1.0e-6);
                    const double sg = sqrt(mrad * mrad + pix * pix * 0.25);
                    const double sg2 = sg * sg;
                    if (th2 > 16.0 * sg2) continue;
                    const double psf = star_psf(th2, sg, sg2, pix, s, dxm, dym, mprof);
                    const double lum = (0.5 + 1.5 * unit(mh + 29ULL)) * s.cluster_member_brightness;
                    float tint[3];
                    star_tint(cl(unit(mh + 43ULL) + s.star_temperature_bias * 0.4, 0.0, 1.0), s.star_color_variation, tint);
                    const double f = lum * psf;
                    acc[0] += f * static_cast<double>(tint[0]) * static_cast<double>(s.cluster_core_tint[0]);
                    acc[1] += f * static_cast<double>(tint[1]) * static_cast<double>(s.cluster_core_tint[1]);
                    acc[2] += f * static_cast<double>(tint[2]) * static_cast<double>(s.cluster_core_tint[2]);
                }
            }
        }
    }
}

// Interstellar dust (:1320-1345).
RT_SKY_HD void dust(const V3& dir, const SkyProfile& s, double* acc) {
    if (!s.dust_enabled || s.dust_intensity <= 0.0) return;
    const float scale = static_cast<float>(cl(s.dust_scale, 0.2, 8.0));
    const int oct = static_cast<int>(cl(s.dust_fractal_octaves, 1u, 6u));
    const float sf = static_cast<float>(s.seed % 4096u) * 0.77f;
    const float dx = static_cast<float>(dir.x), dy = static_cast<float>(dir.y), dz = static_cast<float>(dir.z);
    const float v = fbm(dx * scale + sf, dy * scale - 53.0f, dz * scale + sf * 0.5f, oct, 0.55f);
    const float thr = static_cast<float>(cl(1.0 - 0.2 * s.dust_density, 0.0, 0.95));
    if (v > thr) {
        const float nv = (v - thr) / (1.0f - thr);
        const double lum = static_cast<double>(powf(nv, static_cast<float>(s.dust_contrast))) * s.dust_intensity * 0.35;
        acc[0] += lum * static_cast<double>(s.dust_tint[0]);
        acc[1] += lum * static_cast<double>(s.dust_tint[1]);
        acc[2] += lum * static_cast<double>(s.dust_tint[2]);
    }
}

// Grid resolution and presence threshold of the sparse point layers.
RT_SKY_HD double sparse_res(double density) { return cl(6.0 * sqrt(cl(density, 0.01, 10.0)), 4.0, 36.0); }

// Quasars with relativistic jets (:1347-1413).
RT_SKY_HD_NOINLINE void quasars(const V3& dir, const SkyProfile& s, double* acc) {
    if (!s.quasar_enabled || s.quasar_density <= 0.0) return;
    const uint64_t seed = static_cast<uint64_t>(s.seed) ^ 0x9b05688c2b3e6c1fULL;
    const double res = sparse_res(s.quasar_density);
    const int32_t cx = static_cast<int32_t>(floor(dir.x * res)), cy = static_cast<int32_t>(floor(dir.y * res)),
                  cz = static_cast<int32_t>(floor(dir.z * res));
    const double presence = cl(1.0 - s.quasar_density * 0.06, 0.05, 0.99);
    #pragma unroll 1
    for (int32_t dz = -1; dz <= 1; ++dz)
        #pragma unroll 1
        for (int32_t dy = -1; dy <= 1; ++dy)
            #pragma unroll 1
            for (int32_t dx = -1; dx <= 1; ++dx) {
                const uint64_t h = hash_3d(cx + dx, cy + dy, cz + dz, seed);
                if (unit(h) <= presence) continue;
                V3 qd;
                if (!cell_point(cx + dx, cy + dy, cz + dz, h, qd)) continue;
                const double mu = dot(dir, qd);
                if (mu <= 0.985) continue;
                const double sep2 = 2.0 * mx(0.0, 1.0 - mu);
                // outside the window the quasar adds exactly zero: skip its jet
                const double support = mx(mx(s.quasar_jet_length, 0.005) * 2.0, mx(s.quasar_core_size, 0.0001) * 8.0);
                if (1.0 - sep2 / (support * support) <= 0.0) continue;
                const double jt = unit(h + 41ULL) * kPi, jp = unit(h + 47ULL) * kTwoPi;
                const double st = m_sin(jt);
                const V3 jet{st * m_cos(jp), st * m_sin(jp), m_cos(jt)};
                const double cv = fabs(dot(dir, jet));
                const double gamma = mx(s.quasar_jet_lorentz_factor, 1.05);
                const double beta = sqrt(1.0 - 1.0 / (gamma * gamma));
                const double dop = 1.0 / (gamma * (1.0 - beta * cv));
                const double boost = m_pow(cl(dop, 0.1, 10.0), 3.0);
                const double core_r = mx(s.quasar_core_size, 0.0001);
                const double core = m_exp(-sep2 / (2.0 * core_r * core_r)) * s.quasar_brightness * 1.5;
                const V3 d{dir.x - qd.x, dir.y - qd.y, dir.z - qd.z};
                const double along = dot(d, jet);
                const double perp2 = mx(sep2 - along * along, 0.0);
                const double jlen = mx(s.quasar_jet_length, 0.005);
                const double open = mx(s.quasar_jet_opening_angle_deg, 1.0) * (kPi / 180.0);
                const double jw = core_r + fabs(along) * m_tan(open);
                const double prof = m_exp(-perp2 / (2.0 * jw * jw)) * m_exp(-fabs(along) / jlen);
                const double knot = 0.8 + 0.2 * m_cos(fabs(along) * 160.0);
                const double jf = prof * knot * s.quasar_jet_intensity * s.quasar_brightness * boost * 0.4;
                const double win = cl(1.0 - sep2 / (support * support), 0.0, 1.0);
                const double t = (core + jf) * win * win;
                acc[0] += t * 0.90;
                acc[1] += t * 1.10;
                acc[2] += t * 1.60;
            }
}

// Pulsars: swept beams and wind nebulae (:1415-1501).
RT_SKY_HD_NOINLINE void pulsars(const V3& dir, const SkyProfile& s, double time, double* acc) {
    if (!s.pulsar_enabled || s.pulsar_brightness <= 0.0) return;
    const uint64_t seed = static_cast<uint64_t>(s.seed) ^ 0x4f1bbcdcu;
    const double res = sparse_res(s.pulsar_density);
    const int32_t cx = static_cast<int32_t>(floor(dir.x * res)), cy = static_cast<int32_t>(floor(dir.y * res)),
                  cz = static_cast<int32_t>(floor(dir.z * res));
    const double presence = cl(1.0 - s.pulsar_density * 0.06, 0.05, 0.99);
    #pragma unroll 1
    for (int32_t dz = -1; dz <= 1; ++dz)
        #pragma unroll 1
        for (int32_t dy = -1; dy <= 1; ++dy)
            #pragma unroll 1
            for (int32_t dx = -1; dx <= 1; ++dx) {
                const uint64_t h = hash_3d(cx + dx, cy + dy, cz + dz, seed);
                if (unit(h) <= presence) continue;
                V3 pd;
                if (!cell_point(cx + dx, cy + dy, cz + dz, h, pd)) continue;
                const double mu = dot(dir, pd);
                if (mu <= 0.996) continue;
                const double sep2 = 2.0 * mx(0.0, 1.0 - mu);
                const double at = unit(h + 49ULL) * kPi, ap = unit(h + 53ULL) * kTwoPi;
                const double sst = m_sin(at);
                const V3 axis{sst * m_cos(ap), sst * m_sin(ap), m_cos(at)};
                const double tilt = s.pulsar_magnetic_tilt_deg * (kPi / 180.0);
                const double jitter = m_exp((unit(h + 83ULL) - 0.5) * s.pulsar_frequency_spread * 2.0);
                const double rate = s.pulsar_pulse_rate * jitter;
                const double phase = m_fmod(time * rate + unit(h + 61ULL), 1.0) * kTwoPi;
                V3 u1, u2;
                tangents(axis, u1, u2);
                const double sti = m_sin(tilt), cti = m_cos(tilt), cph = m_cos(phase), sph = m_sin(phase);
                const V3 beam{cti * axis.x + sti * (cph * u1.x + sph * u2.x), cti * axis.y + sti * (cph * u1.y + sph * u2.y),
                              cti * axis.z + sti * (cph * u1.z + sph * u2.z)};
                const double mub = fabs(dot(dir, beam));
                const double bw = mx(s.pulsar_beam_width_deg, 0.5) * (kPi / 180.0);
                const double bsep2 = 2.0 * mx(0.0, 1.0 - mub);
                const double duty = m_exp(-bsep2 / (2.0 * bw * bw));
                const double core_r = 0.0004;
                const double core = m_exp(-sep2 / (2.0 * core_r * core_r)) * s.pulsar_brightness * 1.8;
                const double pw = mx(s.pulsar_wind_nebula_scale, 0.0005);
                const V3 d{dir.x - pd.x, dir.y - pd.y, dir.z - pd.z};
                const double along = dot(d, axis);
                const double perp2 = mx(sep2 - along * along, 0.0);
                const double torus = m_exp(-perp2 / (2.0 * pw * pw)) * m_exp(-fabs(along) / (pw * 0.4));
                const double pwn = torus * s.pulsar_wind_nebula_intensity * s.pulsar_brightness * 0.5;
                const double t = core * duty + pwn;
                acc[0] += t * 0.70;
                acc[1] += t * 1.30;
                acc[2] += t * 1.15;
            }
}

// Supernova remnants: perturbed shells with interior glow (:1503-1590).
RT_SKY_HD_NOINLINE void remnants(const V3& dir, const SkyProfile& s, double* acc) {
    if (!s.snr_enabled || s.snr_brightness <= 0.0) return;
    const uint64_t seed = static_cast<uint64_t>(s.seed) ^ 0x7a31b9efu;
    const double res = sparse_res(s.snr_density);
    const int32_t cx = static_cast<int32_t>(floor(dir.x * res)), cy = static_cast<int32_t>(floor(dir.y * res)),
                  cz = static_cast<int32_t>(floor(dir.z * res));
    const double presence = cl(1.0 - s.snr_density * 0.06, 0.05, 0.99);
    #pragma unroll 1
    for (int32_t dz = -1; dz <= 1; ++dz)
        #pragma unroll 1
        for (int32_t dy = -1; dy <= 1; ++dy)
            #pragma unroll 1
            for (int32_t dx = -1; dx <= 1; ++dx) {
                const uint64_t h = hash_3d(cx + dx, cy + dy, cz + dz, seed);
                if (unit(h) <= presence) continue;
                V3 sd;
                if (!cell_point(cx + dx, cy + dy, cz + dz, h, sd)) continue;
                const double mu = dot(dir, sd);
                if (mu <= 0.992) continue;
                const double sep2 = 2.0 * mx(0.0, 1.0 - mu);
                const double morph = unit(h + 67ULL);
                const double ex = unit(h + 71ULL) - 0.5, ey = unit(h + 73ULL) - 0.5, ez = unit(h + 79ULL) - 0.5;
                const double el = mx(sqrt(ex * ex + ey * ey + ez * ez), 1.0e-6);
                const double proj = ((dir.x - sd.x) * ex + (dir.y - sd.y) * ey + (dir.z - sd.z) * ez) / el;
                const double es = 1.0 + (morph - 0.5) * s.snr_morphology_variety * 1.1;
                const double base = mx(s.snr_size * (0.8 + 0.4 * s.snr_expansion_age) * es, 0.003);
                const double dist = sqrt(mx(sep2 + proj * proj * (es * es - 1.0), 0.0));
                if (dist > base * 2.2) continue;
                const float turb = fbm(static_cast<float>(dir.x * s.snr_filament_scale * 30.0),
                                       static_cast<float>(dir.y * s.snr_filament_scale * 30.0),
                                       static_cast<float>(dir.z * s.snr_filament_scale * 30.0), 3, 0.6f);
                const double pr = base * (1.0 + s.snr_asymmetry * 0.35 * static_cast<double>(turb));
                const double thick = mx(s.snr_shell_thickness * base, 0.0005);
                const double diff = fabs(dist - pr);
                const double shell = m_exp(-(diff * diff) / (2.0 * thick * thick)) * s.snr_brightness * 1.5;
                const double boost = (morph > 0.5) ? 1.6 : 0.4;
                const double inner = (dist < pr) ? (m_exp(-dist / pr) * s.snr_interior_glow * s.snr_brightness * boost) : 0.0;
                const double maxr = base * 1.6;
                const double win = cl(1.0 - sep2 / (maxr * maxr), 0.0, 1.0);
                const double herm = win * win;
                double vs[3], vi[3];
                const double cs = unit(h + 83ULL);
                if (cs < 0.33) {
                    vs[0] = 0.45; vs[1] = 1.45; vs[2] = 1.05; vi[0] = 0.25; vi[1] = 0.85; vi[2] = 1.45;
                } else if (cs < 0.66) {
                    vs[0] = 1.65; vs[1] = 0.40; vs[2] = 0.55; vi[0] = 1.35; vi[1] = 0.70; vi[2] = 0.30;
                } else {
                    vs[0] = 1.45; vs[1] = 1.15; vs[2] = 0.35; vi[0] = 0.95; vi[1] = 0.40; vi[2] = 1.35;
                }
                const double cv = cl(s.snr_color_variation, 0.0, 2.0);
                for (int k = 0; k < 3; ++k) {
                    const double sc = static_cast<double>(s.snr_shell_color[k]) * (1.0 - 0.5 * cv) + vs[k] * 0.5 * cv;
                    const double ic = static_cast<double>(s.snr_interior_color[k]) * (1.0 - 0.5 * cv) + vi[k] * 0.5 * cv;
                    acc[k] += (shell * sc + inner * ic) * herm;
                }
            }
}

// Celestial coordinate grid and cell fills (:528-668); returns the alpha.
RT_SKY_HD_NOINLINE double grid(const V3& dir, const SkyProfile& s, double fov, double* col) {
    col[0] = col[1] = col[2] = 0.0;
    if (!s.grid_enabled || (s.grid_opacity <= 0.0 && s.grid_cell_opacity <= 0.0)) return 0.0;
    const double dec = m_asin(cl(dir.z, -1.0, 1.0));
    const double ra = m_atan2(dir.y, dir.x);
    const double sp = mx(s.grid_spacing_deg, 0.1) * kDegToRad;
    const double pix = mx(fov / 1080.0, 1.0e-7);
    const double cdec = mx(m_cos(dec), 1.0e-6);
    double alpha = 0.0;
    if (s.grid_cell_fill_mode != 0u && s.grid_cell_opacity > 0.0) {
        const double ds = dec + kHalfPi;
        const double rs = (ra < 0.0) ? (ra + kTwoPi) : ra;
        const int32_t cd = static_cast<int32_t>(floor(ds / sp)), cr = static_cast<int32_t>(floor(rs / sp));
        const int32_t nc = cl(static_cast<int32_t>(s.grid_cell_color_count), 1, 16);
        int32_t pick = 0;
        if (s.grid_cell_fill_mode == 1u) {
            pick = ((cd + cr) % 2 + 2) % 2;
        } else if (s.grid_cell_fill_mode == 2u) {
            pick = ((cd + 2 * cr) % nc + nc) % nc;
        } else if (s.grid_cell_fill_mode == 3u) {
            pick = (((cr % 2 + 2) % 2) + 2 * ((cd % 2 + 2) % 2)) % nc;
        } else if (s.grid_cell_fill_mode == 4u) {
            const uint64_t ch = hash_coords(static_cast<uint32_t>(cd + 10000), static_cast<uint32_t>(cr + 10000),
                                            static_cast<uint64_t>(s.seed) ^ 0x5a17ULL);
            pick = static_cast<int32_t>(unit(ch) * static_cast<double>(nc)) % nc;
        }
        col[0] = static_cast<double>(s.grid_cell_colors[pick][0]);
        col[1] = static_cast<double>(s.grid_cell_colors[pick][1]);
        col[2] = static_cast<double>(s.grid_cell_colors[pick][2]);
        alpha = cl(s.grid_cell_opacity, 0.0, 1.0);
    }
    if (s.grid_opacity <= 0.0) return alpha;
    const double fe = mx(pix * 0.6, 1.0e-8);
    const double hw_maj = mx(s.grid_major_width, pix) * 0.5, hw_min = mx(s.grid_minor_width, pix * 0.7) * 0.5;
    const double hw_eq = mx(s.grid_equator_width, pix) * 0.5, hw_pol = mx(s.grid_polar_width, pix) * 0.5;
    const double hw_mer = mx(s.grid_meridian_width, pix) * 0.5, hw_tick = mx(s.grid_tick_width, pix) * 0.5;
    // line coverage at a distance from a line of half width hw
    auto line = [fe](double dist, double hw) { return 1.0 - cl((dist - (hw - fe)) / (2.0 * fe), 0.0, 1.0); };
    const double taper = cl((sp * cdec - hw_maj * 0.5) / mx(hw_maj * 2.5, 1.0e-6), 0.0, 1.0);
    const double d_dec = fabs(m_remainder(dec, sp));
    const double d_ra = fabs(m_remainder(ra, sp)) * cdec;
    const double cov_major = mx(line(d_dec, hw_maj), line(d_ra, hw_maj) * taper);
    double cov_sub = 0.0;
    if (s.grid_subdivisions > 0u) {
        const double ssp = sp / static_cast<double>(s.grid_subdivisions + 1u);
        const double a = line(fabs(m_remainder(dec, ssp)), hw_min);
        const double st = cl((ssp * cdec - hw_min * 0.5) / mx(hw_min * 2.5, 1.0e-6), 0.0, 1.0);
        const double b = line(fabs(m_remainder(ra, ssp)) * cdec, hw_min) * st;
        cov_sub = mx(a, b) * 0.75;
    }
    const double cov_eq = s.grid_show_equator ? line(fabs(dec), hw_eq) * cl(s.grid_equator_opacity, 0.0, 1.0) : 0.0;
    const double cov_pm = s.grid_show_meridians
                              ? line(fabs(m_remainder(ra, kPi)) * cdec, hw_mer) * taper * cl(s.grid_meridian_opacity, 0.0, 1.0)
                              : 0.0;
    const double cov_cap = s.grid_show_polar_caps
                               ? line(fabs(fabs(dec) - (kHalfPi - sp)), hw_pol) * cl(s.grid_polar_opacity, 0.0, 1.0)
                               : 0.0;
    double cov_ticks = 0.0;
    if (s.grid_show_ticks) {
        const double tsp = mx(s.grid_tick_interval_deg, 0.1) * kDegToRad;
        const double ext = mx(s.grid_tick_length, pix * 2.0);
        if (fabs(dec) < ext) {
            const double t = line(fabs(m_remainder(ra, tsp)) * cdec, hw_tick) *
                             (1.0 - cl((fabs(dec) - (ext - fe)) / (2.0 * fe), 0.0, 1.0));
            cov_ticks = mx(cov_ticks, t);
        }
        const double rq = fabs(m_remainder(ra, kHalfPi) * cdec);
        if (rq < ext) {
            const double t = line(fabs(m_remainder(dec, tsp)), hw_tick) * (1.0 - cl((rq - (ext - fe)) / (2.0 * fe), 0.0, 1.0));
            cov_ticks = mx(cov_ticks, t * taper);
        }
    }
    const double gr = mx(hw_maj * 6.0, pix * 4.0);
    const double gdec = m_exp(-d_dec * d_dec / (2.0 * gr * gr));
    const double gra = m_exp(-d_ra * d_ra / (2.0 * gr * gr)) * taper;
    const double glow = mx(gdec, gra) * cl(s.grid_glow, 0.0, 10.0);
    auto layer = [&](double cov, const float* c, double boost) {
        if (cov <= 0.0) return;
        const double a = cl(cov * s.grid_opacity, 0.0, 1.0);
        col[0] = col[0] * (1.0 - a) + static_cast<double>(c[0]) * boost * a;
        col[1] = col[1] * (1.0 - a) + static_cast<double>(c[1]) * boost * a;
        col[2] = col[2] * (1.0 - a) + static_cast<double>(c[2]) * boost * a;
        alpha = alpha + a * (1.0 - alpha);
    };
    layer(cov_sub, s.grid_minor_color, 0.85);
    layer(cov_major, s.grid_major_color, 1.0 + glow);
    layer(cov_cap, s.grid_polar_color, 1.1);
    layer(cov_pm, s.grid_meridian_color, 1.15);
    layer(cov_eq, s.grid_equator_color, 1.2);
    layer(cov_ticks, s.grid_tick_color, 1.3);
    return cl(alpha, 0.0, 1.0);
}

// The sky colour in direction (x, y, z) for a camera of field of view `fov`
// (radians) at time `time` (SkyboxRenderer::sample_sky, :1674-1722, with the
// profile's time replaced by the scene's), for the threads with `active` set;
// `between(layer)` runs after each enabled layer on every thread, active or not (a
// block barrier in the device shading pass, so that the warps of a block run
// one layer's code at a time and share the instruction cache; nothing on the
// host).  The layers follow the profile, so every thread calls between() the
// same number of times.
// The layers in their order, as between() is told which one ended.
enum Layer : int { L_NEBULAE = 0, L_DUST, L_GALAXIES, L_CLUSTERS, L_QUASARS, L_PULSARS, L_REMNANTS, L_STARS };

template <class Between>
RT_SKY_HD void sample_phased(const SkyProfile& s, double x, double y, double z, double fov, double time, bool active,
                             float* out, Between&& between) {
    out[0] = out[1] = out[2] = 0.0f;
    if (!s.enabled) return;
    const double l2 = x * x + y * y + z * z;
    active = active && !(l2 < 1.0e-18);
    V3 d{0.0, 0.0, 0.0}, u{0.0, 0.0, 0.0};
    double acc[3] = {static_cast<double>(s.background_color[0]), static_cast<double>(s.background_color[1]),
                     static_cast<double>(s.background_color[2])};
    if (active) {
        const double inv = 1.0 / sqrt(l2);
        u = V3{x * inv, y * inv, z * inv};
        double yaw = s.orientation_yaw_deg;
        if (s.dynamic_rotation) yaw = m_remainder(yaw + s.rotation_rate_deg_s * time, 360.0);
        d = rotate(u, yaw, s.orientation_pitch_deg, s.orientation_roll_deg);
    }
    const double fov_deg = fov * (180.0 / kPi);
    const double zoom = cl(s.adaptive_fov_reference / mx(fov_deg, 0.05), 1.0, 128.0);
    // the layers that move read the scene's time in place of the profile's
    if (s.nebula_enabled) {
        if (active) nebulae(d, s, zoom, acc);
        between(L_NEBULAE);
    }
    if (s.dust_enabled) {
        if (active) dust(d, s, acc);
        between(L_DUST);
    }
    if (s.galaxies_enabled) {
        if (active) galaxies(d, s, acc);
        between(L_GALAXIES);
    }
    if (s.clusters_enabled) {
        if (active) clusters(d, s, fov, acc);
        between(L_CLUSTERS);
    }
    if (s.quasar_enabled) {
        if (active) quasars(d, s, acc);
        between(L_QUASARS);
    }
    if (s.pulsar_enabled) {
        if (active) pulsars(d, s, time, acc);
        between(L_PULSARS);
    }
    if (s.snr_enabled) {
        if (active) remnants(d, s, acc);
        between(L_REMNANTS);
    }
    if (s.stars_enabled) {
        if (active) stars(d, s, fov, time, acc);
        between(L_STARS);
    }
    if (!active) return;
    const double k = mx(s.master_intensity, 0.0);
    float rgb[3] = {static_cast<float>(mx(0.0, acc[0] * k)), static_cast<float>(mx(0.0, acc[1] * k)),
                    static_cast<float>(mx(0.0, acc[2] * k))};
    hue_saturation(rgb, s.hue_shift_deg * (kPi / 180.0), s.saturation);
    if (s.grid_enabled) {
        const V3 gd = rotate(u, s.grid_orientation_yaw_deg, s.grid_orientation_pitch_deg, s.grid_orientation_roll_deg);
        double gc[3];
        const double a = grid(gd, s, fov, gc);
        if (a > 0.0)
            for (int i = 0; i < 3; ++i) rgb[i] = static_cast<float>(static_cast<double>(rgb[i]) * (1.0 - a) + gc[i] * a);
    }
    out[0] = rgb[0];
    out[1] = rgb[1];
    out[2] = rgb[2];
}

// The sky colour of one direction (sample_phased for a lone thread).
RT_SKY_HD_NOINLINE void sample(const SkyProfile& s, double x, double y, double z, double fov, double time, float* out) {
    sample_phased(s, x, y, z, fov, time, true, out, [](int) {});
}

}  // namespace sky
}  // namespace relsim
