// ref_shade_driver.cpp -- C entry points over the UNMODIFIED reference's
// pixel shading: the primary disk profile (AccretionDiskModel::
// resolve_primary_profile / finalize), thin-disk shading (AccretionDiskModel::
// shade, and HydroDiskShader's Novikov-Thorne context for hydro model 1),
// blackbody colour (blackbody_linear_rgb) and SoftwareComputeEngine::
// apply_tonemapping, which the reference declares private.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into
// oracle/_ref/libref_oracle.so.  To reach the private static member without
// editing the reference, this translation unit makes `private` expand to
// `public` while it includes the engine header (the standard headers are
// included first, unaffected).
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <functional>
#include <future>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numbers>
#include <numeric>
#include <optional>
#include <random>
#include <span>
#include <sstream>
#include <string>
#include <string_view>
#include <thread>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <variant>
#include <vector>

#define private public
#include "relativistic/render/software_compute_engine.hpp"
#undef private

namespace R = Relativistic::Render;

static R::GpuDiskProfile profile_from(const float p[32]) {
	R::GpuDiskProfile d{};
	static_assert(sizeof(R::GpuDiskProfile) == 32 * sizeof(float));
	std::memcpy(&d, p, sizeof d);
	return d;
}

extern "C" {

// resolve_primary_profile: the push constants' temperatures, saturation and
// beaming override the profile, then finalize (clamps, temperature
// normalisation, reference luminance).  in: disk_temperature_scale_k,
// disk_temperature_floor_k, disk_color_saturation, disk_doppler_beaming_exponent.
void ref_resolve_profile(const float profile[32], const double in[4], float out[32]) {
	R::GpuCameraPushConstants p{};
	p.primary_disk = profile_from(profile);
	p.disk_temperature_scale_k = in[0];
	p.disk_temperature_floor_k = in[1];
	p.disk_color_saturation = in[2];
	p.disk_doppler_beaming_exponent = in[3];
	const R::GpuDiskProfile r = R::AccretionDiskModel::resolve_primary_profile(p);
	std::memcpy(out, &r, sizeof r);
}

// Thin-disk radiance and opacity at one surface point.  hydro_model 0: the
// procedural temperature profile (AccretionDiskModel::shade); 1: the
// Novikov-Thorne flux profile (HydroDiskShader::context(...).shade_thin_disk).
// point: mass, spin, inner, outer, radius, azimuth, redshift, time, detail.
// out: r, g, b, opacity.
void ref_disk_shade(const float profile[32], const double point[9], uint32_t hydro_model, float accretion_rate_scale,
                    double out[4]) {
	const R::GpuDiskProfile d = profile_from(profile);
	R::DiskSurfacePoint pt{};
	pt.mass = point[0];
	pt.spin = point[1];
	pt.inner_radius = point[2];
	pt.outer_radius = point[3];
	pt.radius = point[4];
	pt.azimuth = point[5];
	pt.redshift = point[6];
	pt.time = point[7];
	pt.detail_scale = point[8];
	R::DiskShadingResult s;
	if (hydro_model == 1u) {
		R::GpuHydroDiskProfile h{};
		h.model = 1u;
		h.accretion_rate_scale = accretion_rate_scale;
		const auto& ctx = R::HydroDiskShader::context(h, pt.mass, pt.spin, pt.inner_radius, pt.outer_radius);
		s = ctx.shade_thin_disk(d, pt);
	} else {
		s = R::AccretionDiskModel::shade(d, pt);
	}
	out[0] = s.radiance[0];
	out[1] = s.radiance[1];
	out[2] = s.radiance[2];
	out[3] = s.opacity;
}

// Novikov-Thorne context constants: flux peak over the disk and rate factor.
void ref_nt_context(double mass, double spin, double inner, double outer, float accretion_rate_scale, double out[2]) {
	R::GpuHydroDiskProfile h{};
	h.model = 1u;
	h.accretion_rate_scale = accretion_rate_scale;
	const auto& ctx = R::HydroDiskShader::context(h, mass, spin, inner, outer);
	out[0] = ctx.thin_disk_flux_peak();
	out[1] = ctx.thin_disk_rate_factor();
}

void ref_blackbody_rgb(double temperature_k, double reference_luminance, double out[3]) {
	const auto c = R::AccretionDiskModel::blackbody_linear_rgb(temperature_k, reference_luminance);
	out[0] = c[0];
	out[1] = c[1];
	out[2] = c[2];
}

// The procedural sky (SkyboxRenderer::sample_sky) in direction (x, y, z) for
// a GpuSkyProfile image (1808 bytes), a field of view and a scene time.
void ref_sample_sky(const void* profile, double x, double y, double z, double fov, double time, float out[3]) {
	R::GpuSkyProfile p;
	std::memcpy(&p, profile, sizeof p);
	const auto c = R::SkyboxRenderer::sample_sky(x, y, z, p.to_settings(), fov, time);
	out[0] = c[0];
	out[1] = c[1];
	out[2] = c[2];
}

// The default GpuSkyProfile image.
void ref_sky_profile_defaults(void* out) {
	const R::GpuSkyProfile p{};
	std::memcpy(out, &p, sizeof p);
}

// Hydro model 2: the reference's HydroDiskContext for the Fishbone-Moncrief
// torus (hydro_disk_shading.hpp:76-110): out = valid, closed, max enthalpy,
// inner and outer bounds, specific angular momentum, W_in.
static R::GpuHydroDiskProfile hydro_from(const double torus[5]) {
	R::GpuHydroDiskProfile p{};
	p.model = 2;
	p.torus_inner_radius = static_cast<float>(torus[0]);
	p.torus_center_radius = static_cast<float>(torus[1]);
	p.adiabatic_index = static_cast<float>(torus[2]);
	p.optical_depth_scale = static_cast<float>(torus[3]);
	p.sampling_density = static_cast<float>(torus[4]);
	return p;
}

void ref_fm_context(const double torus[5], double mass, double spin, double out[7]) {
	const R::HydroDiskContext c(hydro_from(torus), mass, spin, 6.0 * mass, 24.0 * mass);
	out[0] = c.torus_valid() ? 1.0 : 0.0;
	out[1] = c.torus_closed() ? 1.0 : 0.0;
	out[2] = c.max_enthalpy();
	out[3] = c.torus_inner_bound();
	out[4] = c.torus_outer_bound();
	out[5] = c.torus_specific_angular_momentum();
	out[6] = c.torus_potential_inner();
}

// HydroDiskContext::integrate_segment (:173-269) of one chord with a disk
// profile as it stands: out = radiance r, g, b, opacity, redshift.
void ref_fm_segment(const double torus[5], const float profile[32], double mass, double spin, const double from[3],
                    const double to[3], double l_over_e, double out[5]) {
	const R::HydroDiskContext c(hydro_from(torus), mass, spin, 6.0 * mass, 24.0 * mass);
	const auto s = c.integrate_segment(profile_from(profile), {from[0], from[1], from[2]}, {to[0], to[1], to[2]},
	                                   l_over_e);
	out[0] = s.radiance[0];
	out[1] = s.radiance[1];
	out[2] = s.radiance[2];
	out[3] = s.opacity;
	out[4] = s.redshift;
}

void ref_tonemap(const double rgb[3], uint32_t mode, double exposure_ev, float out[3]) {
	const auto c = R::SoftwareComputeEngine::apply_tonemapping({rgb[0], rgb[1], rgb[2]}, mode, exposure_ev);
	out[0] = c[0];
	out[1] = c[1];
	out[2] = c[2];
}

}  // extern "C"
