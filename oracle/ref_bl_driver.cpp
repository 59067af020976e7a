// ref_bl_driver.cpp -- C entry points over the UNMODIFIED reference's
// Boyer-Lindquist metrics (KerrNewmanMetric, KerrMetric), their analytic
// Christoffel symbols, the ZAMO tetrad and light ray, and an independent trace
// through RK45AdaptiveIntegrator<KerrNewmanMetric>.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into
// oracle/_ref/libref_oracle.so beside ref_driver.cpp; it pins the C
// restatement in bl_oracle.c.
#include "relativistic/core/math/christoffel.hpp"
#include "relativistic/integrators/rk45_adaptive.hpp"
#include "relativistic/integrators/step_controller.hpp"
#include "relativistic/metrics/kerr.hpp"
#include "relativistic/metrics/kerr_newman.hpp"
#include "relativistic/observer/observer_tetrad.hpp"

#include <cmath>
#include <numbers>

namespace C = Relativistic::Core;
namespace M = Relativistic::Metrics;
namespace I = Relativistic::Integrators;
namespace O = Relativistic::Observer;

namespace {

template <typename Metric>
void metric_out(const Metric& metric, const double x[4], double g[16]) {
    const auto gm = metric.metric_tensor(C::FourVector<double>(x[0], x[1], x[2], x[3]));
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) g[4 * i + j] = gm(i, j);
}

// Gamma^mu_ab (analytic, through the reference's compute_christoffel dispatch)
// and the acceleration -Gamma^mu_ab u^a u^b summed over all a, b.
template <typename Metric>
void christoffel_out(const Metric& metric, const double x[4], const double u[4], double gamma[64], double acc[4]) {
    const auto G = C::compute_christoffel<C::DerivativeOrder::EighthOrder, Metric, double>(
        metric, C::FourVector<double>(x[0], x[1], x[2], x[3]));
    for (int mu = 0; mu < 4; ++mu) {
        double s = 0.0;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const double v = G(mu, a, b);
                if (gamma) gamma[16 * mu + 4 * a + b] = v;
                s -= v * u[a] * u[b];
            }
        acc[mu] = s;
    }
}

}  // namespace

extern "C" {

void ref_kn_metric(double mass, double spin, double charge, const double x[4], double g[16]) {
    metric_out(M::KerrNewmanMetric<double>(mass, spin, charge, 1.0, 1.0, 1.0), x, g);
}

void ref_kerr_bl_metric(double mass, double spin, const double x[4], double g[16]) {
    metric_out(M::KerrMetric<double>(mass, spin, 1.0, 1.0), x, g);
}

void ref_kn_christoffel(double mass, double spin, double charge, const double x[4], const double u[4],
                        double gamma[64], double acc[4]) {
    christoffel_out(M::KerrNewmanMetric<double>(mass, spin, charge, 1.0, 1.0, 1.0), x, u, gamma, acc);
}

void ref_kerr_bl_christoffel(double mass, double spin, const double x[4], const double u[4], double gamma[64],
                             double acc[4]) {
    christoffel_out(M::KerrMetric<double>(mass, spin, 1.0, 1.0), x, u, gamma, acc);
}

double ref_kn_horizon(double mass, double spin, double charge) {
    return M::KerrNewmanMetric<double>(mass, spin, charge, 1.0, 1.0, 1.0).outer_horizon_radius();
}

// trace_exact_photon's initial ray (software_compute_engine.hpp:1347-1350):
// ZAMO tetrad at (r, theta, phi), u = construct_light_ray(-n_r, -n_th, -n_ph).
void ref_kn_zamo_ray(double mass, double spin, double charge, double r, double theta, double phi, double n_r,
                     double n_th, double n_ph, double u[4]) {
    const M::KerrNewmanMetric<double> metric(mass, spin, charge, 1.0, 1.0, 1.0);
    const auto tetrad = O::ObserverTetrad<double>::make_zamo(metric, C::FourVector<double>(0.0, r, theta, phi));
    const auto v = tetrad.construct_light_ray(-n_r, -n_th, -n_ph);
    for (int i = 0; i < 4; ++i) u[i] = v(i);
}

// Independent trace through RK45AdaptiveIntegrator<KerrNewmanMetric> (4-D
// Christoffel form, Null, PI30), forwards in lambda from the time-reversed
// ray v = -u, with the pole reflection of software_compute_engine.hpp:1492-1500
// after each step and the step cap of the tracer.  Classification: captured
// r < cap_scale r_+, escaped r > r_esc, disk = first theta = pi/2 crossing
// whose bisected root (each trial one fresh single step from the step's start)
// has r on [r_in, r_out] and r > 1.02 r_+ (r_out <= 0: no disk).
// y0 = (r, theta, phi, u^t, u^r, u^theta, u^phi) with u future-directed.
// out: status, r, theta, phi, r_hit, accepted steps, rejected steps.
void ref_kn_rk45_trace(const double y0[7], double mass, double spin, double charge, double rtol, double atol,
                       double cap_fraction, double cap_scale, double r_esc, double r_in, double r_out, int max_steps,
                       double out[7]) {
    const M::KerrNewmanMetric<double> metric(mass, spin, charge, 1.0, 1.0, 1.0);
    I::RK45Config<double> cfg;
    cfg.rtol = rtol;
    cfg.atol = atol;
    cfg.min_step = 1e-12;
    cfg.max_step = 1e13;
    cfg.step_controller_mode = I::StepControllerMode::PI30;
    cfg.crossing_mode = I::HorizonCrossingMode::Continuity;
    I::RK45AdaptiveIntegrator<M::KerrNewmanMetric<double>, double> integ(metric, I::GeodesicType::Null, cfg);
    const double rh = metric.outer_horizon_radius();
    const double pi = std::numbers::pi_v<double>;
    I::GeodesicState<double> s;
    s.x = C::FourVector<double>(0.0, y0[0], y0[1], y0[2]);
    s.u = C::FourVector<double>(-y0[3], -y0[4], -y0[5], -y0[6]);
    double dt = 0.01 * y0[0];
    double status = 0.0, r_hit = NAN;
    for (int it = 0; it < max_steps; ++it) {
        const double r = s.x(1);
        if (r < cap_scale * rh) { status = 1.0; break; }
        if (r > r_esc) { status = 2.0; break; }
        const double cap = cap_fraction * std::max(r - rh, 0.01 * mass);
        if (dt > cap) dt = cap;
        const auto prev = s;
        const auto taken = integ.step(s, dt);
        if (!taken.has_value()) { status = 1.0; break; }
        const double f0 = prev.x(2) - 0.5 * pi, f1 = s.x(2) - 0.5 * pi;
        if (r_out > 0.0 && f0 * f1 <= 0.0 && f0 != f1) {
            double lo = 0.0, hi = 1.0;
            I::GeodesicState<double> mid = s;
            for (int b = 0; b < 64 && hi - lo > 1e-15; ++b) {
                const double t = 0.5 * (lo + hi);
                auto trial = prev;
                double tdt = t * (*taken);
                I::RK45AdaptiveIntegrator<M::KerrNewmanMetric<double>, double> one(metric, I::GeodesicType::Null, cfg);
                if (!one.step(trial, tdt).has_value()) break;
                mid = trial;
                if ((trial.x(2) - 0.5 * pi > 0.0) == (f0 > 0.0)) lo = t; else hi = t;
            }
            const double rr = mid.x(1);
            if (rr >= r_in && rr <= r_out && rr > 1.02 * rh) {
                status = 3.0;
                r_hit = rr;
                s = mid;
                break;
            }
        }
        if (s.x(2) < 0.0) {
            s.x(2) = -s.x(2);
            s.x(3) += pi;
            s.u(2) = -s.u(2);
        } else if (s.x(2) > pi) {
            s.x(2) = 2.0 * pi - s.x(2);
            s.x(3) += pi;
            s.u(2) = -s.u(2);
        }
    }
    out[0] = status;
    out[1] = s.x(1);
    out[2] = s.x(2);
    out[3] = s.x(3);
    out[4] = r_hit;
    out[5] = static_cast<double>(integ.statistics().accepted_steps);
    out[6] = static_cast<double>(integ.statistics().rejected_steps);
}

}  // extern "C"
