// ref_driver.cpp -- C entry points over the UNMODIFIED reference headers.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the reference
// source tree into oracle/_ref/libref_oracle.so (git-ignored).  It pins the C
// restatement in ks_oracle.c against the reference's own functions, gives the
// reference's CPU image path ("Oracle A", SoftwareComputeEngine::dispatch_fp64)
// for the CPU baseline, and an independent FP64 cross-check through the
// reference's 4-D RK45AdaptiveIntegrator<KerrSchildMetric>.
#include "relativistic/core/kerr_schild_null_integrator.hpp"
#include "relativistic/hydro/novikov_thorne.hpp"
#include "relativistic/integrators/rk45_adaptive.hpp"
#include "relativistic/integrators/step_controller.hpp"
#include "relativistic/metrics/kerr_invariants.hpp"
#include "relativistic/metrics/kerr_schild.hpp"
#include "relativistic/observer/camera_projections.hpp"
#include "relativistic/render/accretion_disk/accretion_disk_model.hpp"
#include "relativistic/render/software_compute_engine.hpp"

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace C = Relativistic::Core;
namespace M = Relativistic::Metrics;
namespace I = Relativistic::Integrators;
namespace R = Relativistic::Render;

extern "C" {

void ref_ks_field(const double x[3], double mass, double spin, double* r, double* h, double k[3]) {
	const auto f = C::kerr_schild_field<double>({x[0], x[1], x[2]}, mass, spin);
	*r = f.r;
	*h = f.h;
	for (int i = 0; i < 3; ++i) k[i] = f.k[i];
}

void ref_ks_rhs(const double y[6], double mass, double spin, double dy[6]) {
	C::KerrSchildNullState<double> s;
	s.position = {y[0], y[1], y[2]};
	s.momentum = {y[3], y[4], y[5]};
	const auto d = C::kerr_schild_null_derivatives(s, mass, spin);
	for (int i = 0; i < 3; ++i) {
		dy[i] = d.position[i];
		dy[3 + i] = d.momentum[i];
	}
}

void ref_ks_rk4_step(double y[6], double h, double mass, double spin) {
	C::KerrSchildNullState<double> s;
	s.position = {y[0], y[1], y[2]};
	s.momentum = {y[3], y[4], y[5]};
	C::step_kerr_schild_null_rk4(s, h, mass, spin);
	for (int i = 0; i < 3; ++i) {
		y[i] = s.position[i];
		y[3 + i] = s.momentum[i];
	}
}

void ref_ks_position_from_bl(double r, double th, double ph, double spin, double out[3]) {
	const auto x = C::kerr_schild_position_from_boyer_lindquist(r, th, ph, spin);
	for (int i = 0; i < 3; ++i) out[i] = x[i];
}

void ref_bl_from_ks(const double x[3], double spin, double prev_phi, double out[3]) {
	const auto p = C::boyer_lindquist_from_kerr_schild<double>({x[0], x[1], x[2]}, spin, prev_phi);
	out[0] = p.r;
	out[1] = p.theta;
	out[2] = p.phi;
}

void ref_initial_momentum(const double x[3], double mass, double spin, const double outward[3], double p[3]) {
	const auto m = C::kerr_schild_initial_momentum<double>({x[0], x[1], x[2]}, mass, spin, {outward[0], outward[1], outward[2]});
	for (int i = 0; i < 3; ++i) p[i] = m[i];
}

double ref_redshift_at(double mass, double spin, double radius, double lz) {
	return R::AccretionDiskModel::redshift_at(mass, spin, radius, lz);
}

double ref_isco_radius(double mass, double spin) {
	Relativistic::Hydro::NovikovThorneConfig<double> cfg;
	cfg.mass = mass;
	cfg.spin_parameter = spin;
	cfg.speed_of_light = 1.0;
	cfg.gravitational_constant = 1.0;
	return Relativistic::Hydro::NovikovThorneDisk<double>(cfg).isco_radius();
}

void ref_pinhole_ray(double u, double v, double fov, double n[3]) {
	const auto d = Relativistic::Observer::CameraProjector<double>::compute_pinhole_ray(u, v, fov);
	for (int i = 0; i < 3; ++i) n[i] = d[i];
}

// Sequence of PI30 factors for a sequence of (err, order_p1) calls.
void ref_pi30_sequence(const double* err, const double* order_p1, int n, double* factor) {
	I::AdaptiveStepController<double> ctl(I::StepControllerMode::PI30);
	for (int i = 0; i < n; ++i) factor[i] = ctl.next_factor(err[i], order_p1[i]);
}

// Contravariant KS 4-velocity of the covector (p_t = -1, p_i).
static C::FourVector<double> contravariant(const M::KerrSchildMetric<double>& metric, const double y[6]) {
	const C::FourVector<double> x(0.0, y[0], y[1], y[2]);
	const auto gi = metric.inverse_metric(x);
	const double p[4] = {-1.0, y[3], y[4], y[5]};
	C::FourVector<double> u(0.0, 0.0, 0.0, 0.0);
	for (int mu = 0; mu < 4; ++mu) {
		double s = 0.0;
		for (int nu = 0; nu < 4; ++nu) s += gi(mu, nu) * p[nu];
		u(mu) = s;
	}
	return u;
}

// Kerr invariants (E, L_z, Q, K, norm) of the KS state through the reference's
// KS -> BL map and compute_kerr_invariants_bl.
void ref_kerr_invariants(const double y[6], double mass, double spin, double out[5]) {
	const M::KerrSchildMetric<double> ks(mass, spin, 1.0, 1.0);
	const M::KerrMetric<double> bl(mass, spin, 1.0, 1.0);
	const C::FourVector<double> x(0.0, y[0], y[1], y[2]);
	const auto u = contravariant(ks, y);
	const auto st = M::kerr_schild_to_boyer_lindquist(ks, x, u);
	const auto q = M::compute_kerr_invariants_bl(bl, st.x, st.u);
	out[0] = q.energy;
	out[1] = q.angular_momentum_z;
	out[2] = q.carter_constant;
	out[3] = q.total_carter_constant;
	out[4] = q.rest_mass_norm;
}

// Independent trace through the reference's RK45AdaptiveIntegrator (4-D
// Christoffel form, Null, PI30).  The ray is integrated forwards in lambda
// from the time-reversed 4-velocity.  Classification mirrors ks_oracle.c:
// captured r < cap_scale r_+, escaped r > r_esc, disk = first z sign change
// whose bisected root has r in [r_in, r_out].
// out: status, r, theta, phi, r_hit, accepted steps, rejected steps.
void ref_rk45_trace(const double y0[6], double mass, double spin, double rtol, double atol, double cap_fraction,
                    double cap_scale, double r_esc, double r_in, double r_out, int max_steps, double out[7]) {
	const M::KerrSchildMetric<double> metric(mass, spin, 1.0, 1.0);
	I::RK45Config<double> cfg;
	cfg.rtol = rtol;
	cfg.atol = atol;
	cfg.min_step = 1e-12;
	cfg.max_step = 1e13;
	cfg.step_controller_mode = I::StepControllerMode::PI30;
	cfg.crossing_mode = I::HorizonCrossingMode::Continuity;
	I::RK45AdaptiveIntegrator<M::KerrSchildMetric<double>, double> integ(metric, I::GeodesicType::Null, cfg);
	const double rh = metric.outer_horizon_radius();
	I::GeodesicState<double> s;
	s.x = C::FourVector<double>(0.0, y0[0], y0[1], y0[2]);
	const auto u = contravariant(metric, y0);
	s.u = C::FourVector<double>(-u(0), -u(1), -u(2), -u(3));
	double dt = 0.01 * metric.boyer_lindquist_r(s.x);
	double status = 0.0, r_hit = NAN;
	double phi = 0.0;
	{
		const auto p = C::boyer_lindquist_from_kerr_schild<double>({y0[0], y0[1], y0[2]}, spin, 0.0);
		phi = p.phi;
	}
	for (int it = 0; it < max_steps; ++it) {
		const double r = metric.boyer_lindquist_r(s.x);
		if (r < cap_scale * rh) { status = 1.0; break; }
		if (r > r_esc) { status = 2.0; break; }
		const double cap = cap_fraction * std::max(r - rh, 0.01 * mass);
		if (dt > cap) dt = cap;
		const auto prev = s;
		const auto taken = integ.step(s, dt);  // returns the accepted step length
		if (!taken.has_value()) { status = 1.0; break; }
		{
			const auto p = C::boyer_lindquist_from_kerr_schild<double>({s.x(1), s.x(2), s.x(3)}, spin, phi);
			phi = p.phi;
		}
		if (r_out > 0.0 && prev.x(3) * s.x(3) <= 0.0 && prev.x(3) != s.x(3)) {
			// bisection on the fraction t of the accepted step, each trial one fresh
			// single step of length t * taken from the step's start
			double lo = 0.0, hi = 1.0;
			I::GeodesicState<double> mid = s;
			for (int b = 0; b < 64 && hi - lo > 1e-15; ++b) {
				const double t = 0.5 * (lo + hi);
				auto trial = prev;
				double tdt = t * (*taken);
				I::RK45AdaptiveIntegrator<M::KerrSchildMetric<double>, double> one(metric, I::GeodesicType::Null, cfg);
				if (!one.step(trial, tdt).has_value()) break;
				mid = trial;
				if ((trial.x(3) > 0.0) == (prev.x(3) > 0.0)) lo = t; else hi = t;
			}
			const double rr = metric.boyer_lindquist_r(mid.x);
			if (rr >= r_in && rr <= r_out && rr > 1.02 * rh) {
				status = 3.0;
				r_hit = rr;
				s = mid;
				break;
			}
		}
	}
	const auto p = C::boyer_lindquist_from_kerr_schild<double>({s.x(1), s.x(2), s.x(3)}, spin, phi);
	out[0] = status;
	out[1] = p.r;
	out[2] = p.theta;
	out[3] = p.phi;
	out[4] = r_hit;
	out[5] = static_cast<double>(integ.statistics().accepted_steps);
	out[6] = static_cast<double>(integ.statistics().rejected_steps);
}

// The reference's own CPU image path (SoftwareComputeEngine::dispatch_fp64)
// for one camera of the given metric type and charge.  Writes status_flags,
// iterations and redshift per pixel; returns wall seconds.
static double dispatch_fp64_metric(const double observer[4], const double e1[4], const double e2[4],
                                   const double e3[4], double fov, double mass, double spin, double charge,
                                   uint32_t metric_type, double escape_radius, double disk_outer, uint32_t width,
                                   uint32_t height, uint32_t max_steps, uint32_t row_offset, uint32_t row_count,
                                   double step_scale, uint32_t* status, uint32_t* iterations, float* redshift) {
	R::GpuCameraPushConstants p{};
	for (int i = 0; i < 4; ++i) {
		p.observer_position[i] = observer[i];
		p.tetrad_e1[i] = e1[i];
		p.tetrad_e2[i] = e2[i];
		p.tetrad_e3[i] = e3[i];
	}
	p.tetrad_e0 = {1.0, 0.0, 0.0, 0.0};
	p.field_of_view_rad = fov;
	p.metric_mass = mass;
	p.metric_spin = spin;
	p.metric_charge = charge;
	p.metric_type = metric_type;
	p.escape_radius = escape_radius;
	p.max_integration_steps = max_steps;
	p.screen_width = width;
	p.screen_height = height;
	p.projection_mode = 0;
	p.render_flags = 0;
	p.dispatch_row_offset = row_offset;
	p.dispatch_row_count = row_count;
	p.primary_disk.enabled = (disk_outer > 0.0) ? 1.0f : 0.0f;
	p.primary_disk.inner_radius_scale = 1.0f;
	p.primary_disk.outer_radius_mass_units = static_cast<float>(disk_outer);
	p.hydro_disk.model = 1;  // Novikov-Thorne
	// heuristic step (software_compute_engine.hpp:1424-1427) scaled for convergence studies
	p.step_size_factor *= step_scale;
	p.min_step_size *= step_scale;
	const size_t rows = (row_count == 0) ? height : row_count;
	std::vector<R::GpuPixelOutput> out(static_cast<size_t>(width) * rows);
	const auto t0 = std::chrono::steady_clock::now();
	R::SoftwareComputeEngine::dispatch_fp64(p, std::span<R::GpuPixelOutput>(out));
	const auto t1 = std::chrono::steady_clock::now();
	for (size_t i = 0; i < out.size(); ++i) {
		if (status) status[i] = out[i].status_flags;
		if (iterations) iterations[i] = out[i].iterations_used;
		if (redshift) redshift[i] = out[i].redshift;
	}
	return std::chrono::duration<double>(t1 - t0).count();
}

// Oracle A: the reference's own CPU image path for a Kerr-Schild camera
// (metric_type 3), heuristic-step RK4, thin Novikov-Thorne disk.
double ref_dispatch_fp64(const double observer[4], const double e1[4], const double e2[4], const double e3[4], double fov,
                         double mass, double spin, double escape_radius, double disk_outer, uint32_t width,
                         uint32_t height, uint32_t max_steps, uint32_t row_offset, uint32_t row_count,
                         uint32_t* status, uint32_t* iterations, float* redshift) {
	return dispatch_fp64_metric(observer, e1, e2, e3, fov, mass, spin, 0.0, 3u, escape_radius, disk_outer, width,
	                            height, max_steps, row_offset, row_count, 1.0, status, iterations, redshift);
}

// The same for a Kerr-Newman camera (metric_type 5): trace_exact_photon with
// KerrNewmanMetric, the ZAMO ray and heuristic-step RK4 on -Gamma u u, its
// step_size_factor and min_step_size multiplied by step_scale (1: as shipped).
double ref_dispatch_fp64_kn(const double observer[4], const double e1[4], const double e2[4], const double e3[4],
                            double fov, double mass, double spin, double charge, double escape_radius,
                            double disk_outer, uint32_t width, uint32_t height, uint32_t max_steps,
                            uint32_t row_offset, uint32_t row_count, double step_scale, uint32_t* status,
                            uint32_t* iterations, float* redshift) {
	return dispatch_fp64_metric(observer, e1, e2, e3, fov, mass, spin, charge, 5u, escape_radius, disk_outer, width,
	                            height, max_steps, row_offset, row_count, step_scale, status, iterations, redshift);
}

}  // extern "C"
