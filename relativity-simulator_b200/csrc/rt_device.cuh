// rt_device.cuh -- device math of the backward null-geodesic tracer.
//
// Kerr-Schild Hamiltonian with p_t = -1 (kerr_schild_null_integrator.hpp:72-114),
// rewritten for the GPU: the 9 partial derivatives of the null vector are never
// formed.  With dk_j/dx_i contracted against p first, the RHS needs one
// reciprocal each of r, r^2 + a^2 and the Kerr-Schild denominator instead of
// 12 divisions; one rsqrt gives both r and 1/r.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace relsim {

// Dormand-Prince 5(4) tableau (rk45_adaptive.hpp:196-203).
struct DP {
    static constexpr double A21 = 1.0 / 5.0;
    static constexpr double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
    static constexpr double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
    static constexpr double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0,
                            A54 = -212.0 / 729.0;
    static constexpr double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0,
                            A64 = 49.0 / 176.0, A65 = -5103.0 / 18656.0;
    static constexpr double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0, B5 = -2187.0 / 6784.0,
                            B6 = 11.0 / 84.0;
    static constexpr double E1 = 71.0 / 57600.0, E3 = -71.0 / 16695.0, E4 = 71.0 / 1920.0,
                            E5 = -17253.0 / 339200.0, E6 = 22.0 / 525.0, E7 = -1.0 / 40.0;
    // Continuous extension of order 4 (Shampine's dense output for this pair, as
    // in Hairer, Norsett & Wanner, Solving ODEs I, sec. II.6): with
    // d = y1 - y0, b = h k1 - d, c = d - h k7 - b and e = h sum_j D_j k_j,
    // y(t) = y0 + t (d + (1 - t) (b + t (c + (1 - t) e))), t in [0, 1].
    static constexpr double D1 = -12715105075.0 / 11282082432.0, D3 = 87487479700.0 / 32700410799.0,
                            D4 = -10690763975.0 / 1880347072.0, D5 = 701980252875.0 / 199316789632.0,
                            D6 = -1453857185.0 / 822651844.0, D7 = 69997945.0 / 29380423.0;
};

template <typename T>
__device__ __forceinline__ T rt_rsqrt(T v);
template <>
__device__ __forceinline__ double rt_rsqrt<double>(double v) { return rsqrt(v); }
template <>
__device__ __forceinline__ float rt_rsqrt<float>(float v) { return rsqrtf(v); }

template <typename T>
__device__ __forceinline__ T rt_rcp(T v);
template <>
__device__ __forceinline__ double rt_rcp<double>(double v) { return 1.0 / v; }
template <>
__device__ __forceinline__ float rt_rcp<float>(float v) { return __fdividef(1.0f, v); }  // MUFU rcp

template <typename T>
__device__ __forceinline__ T rt_sqrt(T v);
template <>
__device__ __forceinline__ double rt_sqrt<double>(double v) { return sqrt(v); }
template <>
__device__ __forceinline__ float rt_sqrt<float>(float v) {  // MUFU rsqrt based
    const float w = fmaxf(v, 1e-30f);
    return w * rsqrtf(w);
}

// Boyer-Lindquist r of a Kerr-Schild point (kerr_schild_null_integrator.hpp:32-36).
template <typename T>
__device__ __forceinline__ T bl_r2(T x, T y, T z, T a2) {
    const T z2 = z * z;
    const T diff = x * x + y * y + z2 - a2;
    const T r2 = T(0.5) * (diff + rt_sqrt<T>(diff * diff + T(4) * a2 * z2));
    return fmax(r2, T(1e-24));
}

// Hamiltonian RHS.  y = (x, y, z, p_x, p_y, p_z); returns r_BL and, through
// hf/s, the Kerr-Schild scalar H and s = 1 + k.p at y.
//   dx/dl = p - 2 H s k
//   dp/dl = s^2 dH/dx + 2 H s (dk/dx . p)
// with dk/dx_i . p = dr_i * A + B_i (A, B below) and dH/dx_i = C dr_i (+ D for z).
// With GRAV = true the position part returns only the gravitational term
// -2 H s k (the mixed-precision step keeps the free-streaming p in FP64).
template <typename T, bool GRAV = false>
__device__ __forceinline__ T ks_rhs(const T* __restrict__ y, T M, T a, T* __restrict__ dy, T& hf, T& s) {
    const T x = y[0], yy = y[1], z = y[2], px = y[3], py = y[4], pz = y[5];
    const T a2 = a * a;
    const T z2 = z * z;
    const T r2 = bl_r2<T>(x, yy, z, a2);
    const T inv_r = rt_rsqrt<T>(r2);
    const T r = r2 * inv_r;
    const T rpa = r2 + a2;
    const T r4 = r2 * r2;
    const T den = r4 + a2 * z2;
    T inv_rpa, inv_den;
    if constexpr (sizeof(T) == 8) {
        // one reciprocal for both denominators (r^6 stays far from overflow in FP64)
        const T q = rt_rcp<T>(rpa * den);
        inv_rpa = den * q;
        inv_den = rpa * q;
    } else {
        inv_rpa = rt_rcp<T>(rpa);
        inv_den = rt_rcp<T>(den);
    }
    const T r3 = r2 * r;
    const T H = M * r3 * inv_den;
    const T k0 = (r * x + a * yy) * inv_rpa;
    const T k1 = (r * yy - a * x) * inv_rpa;
    const T k2 = z * inv_r;
    const T sv = T(1) + k0 * px + k1 * py + k2 * pz;
    const T two_hs = T(2) * H * sv;
    if constexpr (GRAV) {
        dy[0] = -two_hs * k0;
        dy[1] = -two_hs * k1;
        dy[2] = -two_hs * k2;
    } else {
        dy[0] = px - two_hs * k0;
        dy[1] = py - two_hs * k1;
        dy[2] = pz - two_hs * k2;
    }
    const T r3d = r3 * inv_den;
    const T dr0 = r3d * x;
    const T dr1 = r3d * yy;
    const T dr2 = r * rpa * z * inv_den;
    // C = M r^2 (3 a^2 z^2 - r^4) / den^2 and D = -2 M a^2 r^3 z / den^2, grouped so
    // that FP32 intermediates stay near M / r^2 (no underflow of 1/den^2)
    const T mr2d = M * r2 * inv_den;
    const T C = mr2d * ((T(3) * a2 * z2 - r4) * inv_den);
    const T D = T(-2) * (M * r3 * inv_den) * (a2 * z * inv_den);
    const T A = inv_rpa * ((x - T(2) * r * k0) * px + (yy - T(2) * r * k1) * py) - inv_r * k2 * pz;
    const T B0 = inv_rpa * (r * px - a * py);
    const T B1 = inv_rpa * (r * py + a * px);
    const T B2 = inv_r * pz;
    const T s2 = sv * sv;
    const T G = s2 * C + two_hs * A;
    dy[3] = dr0 * G + two_hs * B0;
    dy[4] = dr1 * G + two_hs * B1;
    dy[5] = dr2 * G + two_hs * B2 + s2 * D;
    hf = H;
    s = sv;
    return r;
}

__device__ __forceinline__ double clampd(double v, double lo, double hi) { return fmin(fmax(v, lo), hi); }

// Disk redshift of a circular orbit (accretion_disk_model.hpp:205-225).
__device__ inline double disk_redshift(double M, double a, double r, double lz) {
    const double am = fabs(a);
    const double sm = sqrt(fmax(M, 1e-12));
    const double sr = sqrt(fmax(r, 1e-12));
    const double r15 = r * sr;
    const double ang = sm / (r15 + am * sm);
    const double bracket = fmax(r15 - 3.0 * M * sr + 2.0 * am * sm, 1e-9);
    const double omega = (a < 0.0) ? -ang : ang;
    const double ut = (r15 + am * sm) / (sqrt(r15) * sqrt(bracket));
    const double den = ut * (1.0 - omega * lz);
    return (fabs(den) > 1e-9) ? clampd(1.0 / den, 0.05, 4.0) : 1.0;
}

// Signed distance of (xi, eta) from the critical curve of a Kerr (q2 = 0) or
// Kerr-Newman hole, in impact parameter (units of M): the smallest local
// minimum R_min of the radial quartic
//   R(r) = (r^2 + a^2 - a xi)^2 - Delta (eta + (xi - a)^2)
//        = r^4 + P r^2 + Qc r + R0,  Delta = r^2 - 2 M r + a^2 + q2
// (carter_ray_classifier.hpp:132-135 for q2 = 0) outside r_+ is moved to zero
// by d_eta = R_min / Delta.  > 0: no turning point.
static __device__ __noinline__ double shadow_distance(double M, double a, double q2, double rh, double xi,
                                                      double eta) {
    const double a2 = a * a;
    const double K = eta + (xi - a) * (xi - a);
    const double P = a2 - xi * xi - eta;
    const double Qc = 2.0 * M * K;
    const double R0 = -a2 * eta - q2 * K;
    const double pp = 0.5 * P, qq = 0.25 * Qc;
    double best = INFINITY, best_r = 0.0;
    auto consider = [&](double r) {
        if (!(r > rh)) return;
        if (12.0 * r * r + 2.0 * P <= 0.0) return;
        const double R = ((r * r + P) * r + Qc) * r + R0;
        if (R < best) {
            best = R;
            best_r = r;
        }
    };
    const double disc = -(4.0 * pp * pp * pp + 27.0 * qq * qq);
    if (disc > 0.0 && pp < 0.0) {
        const double m2 = 2.0 * sqrt(-pp / 3.0);
        const double arg = clampd(3.0 * qq / (pp * m2), -1.0, 1.0);
        const double th = acos(arg) / 3.0;
        constexpr double kThird = 2.0 * 3.14159265358979323846 / 3.0;
        consider(m2 * cos(th));
        consider(m2 * cos(th - kThird));
        consider(m2 * cos(th - 2.0 * kThird));
    } else {
        const double sq = sqrt(fmax(qq * qq / 4.0 + pp * pp * pp / 27.0, 0.0));
        consider(cbrt(-qq / 2.0 + sq) + cbrt(-qq / 2.0 - sq));
    }
    if (!isfinite(best)) return INFINITY;
    const double delta = best_r * best_r - 2.0 * M * best_r + a2 + q2;
    const double b = sqrt(fmax(eta + xi * xi, 1e-30));
    return best / fmax(delta, 1e-30) / (2.0 * b);
}

// Cubic Hermite interpolant of a step from its end points and FSAL slopes.
__device__ __forceinline__ void hermite(const double* y0, const double* f0, const double* y1, const double* f1,
                                        double h, double t, int n, double* out) {
    const double t2 = t * t, t3 = t2 * t;
    const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + t;
    const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
    for (int i = 0; i < n; ++i) out[i] = h00 * y0[i] + h10 * h * f0[i] + h01 * y1[i] + h11 * h * f1[i];
}

// Fraction of the step where the interpolated r_BL crosses `target`
// (Illinois regula falsi; 1 when the end points do not bracket it).
static __device__ double crossing_fraction(const double* y0, const double* f0, const double* y1, const double* f1, double h,
                                    double a, double target) {
    const double a2 = a * a;
    double lo = 0.0, hi = 1.0;
    double flo = sqrt(bl_r2<double>(y0[0], y0[1], y0[2], a2)) - target;
    double fhi = sqrt(bl_r2<double>(y1[0], y1[1], y1[2], a2)) - target;
    if (!((flo > 0.0) != (fhi > 0.0))) return 1.0;
    int side = 0;
    double t = 1.0, x[3];
    for (int it = 0; it < 60; ++it) {
        t = (lo * fhi - hi * flo) / (fhi - flo);
        if (!(t > lo && t < hi)) t = 0.5 * (lo + hi);
        hermite(y0, f0, y1, f1, h, t, 3, x);
        const double ft = sqrt(bl_r2<double>(x[0], x[1], x[2], a2)) - target;
        if (ft == 0.0 || fabs(hi - lo) < 1e-15 || fabs(ft) < 1e-13 * target) break;
        if ((ft > 0.0) == (fhi > 0.0)) {
            hi = t;
            fhi = ft;
            if (side == -1) flo *= 0.5;
            side = -1;
        } else {
            lo = t;
            flo = ft;
            if (side == 1) fhi *= 0.5;
            side = 1;
        }
    }
    return t;
}

// Boyer-Lindquist (r, theta, phi) of a Kerr-Schild point, as Cartesian
// (r sin th cos ph, r sin th sin ph, r cos th): the points the reference's image
// path hands to its volume tests (boyer_lindquist_from_kerr_schild and
// spherical_to_cartesian, software_compute_engine.hpp:1063-1066).
__device__ __forceinline__ void bl_cartesian(const double* x, double a, double* out) {
    const double r = sqrt(bl_r2<double>(x[0], x[1], x[2], a * a));
    const double rho = sqrt(fmax(r * r - x[2] * x[2], 0.0));
    const double th = atan2(rho, x[2]);
    const double ph = atan2(x[1], x[0]) - atan2(a, r);
    const double st = sin(th);
    out[0] = r * st * cos(ph);
    out[1] = r * st * sin(ph);
    out[2] = r * cos(th);
}

// PI30 factor (step_controller.hpp:51-58) from base-2 logs of the errors.
__device__ __forceinline__ float pi30_factor(float le, float lp, float order_p1) {
    return exp2f(-(0.7f / order_p1) * le + (0.3f / order_p1) * (lp - le));
}


// Kerr-Schild field only (r, H, k) at x.
__device__ __forceinline__ double ks_field64(const double* x, double M, double a, double* k, double& hf) {
    const double a2 = a * a;
    const double r2 = bl_r2<double>(x[0], x[1], x[2], a2);
    const double inv_r = rsqrt(r2);
    const double r = r2 * inv_r;
    const double rpa = r2 + a2;
    const double den = r2 * r2 + a2 * x[2] * x[2];
    const double q = 1.0 / (rpa * den);
    const double inv_rpa = den * q;
    hf = M * r2 * r * (rpa * q);
    k[0] = (r * x[0] + a * x[1]) * inv_rpa;
    k[1] = (r * x[1] - a * x[0]) * inv_rpa;
    k[2] = x[2] * inv_r;
    return r;
}

}  // namespace relsim
