// ref_ms_driver.cpp -- C entry points over the UNMODIFIED reference's
// multi-source functions (SoftwareComputeEngine::build_multi_source_data,
// ms_rhs, ms_initial_momentum, ms_inside_horizon), which the reference declares
// private.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into
// oracle/_ref/libref_oracle.so beside ref_driver.cpp.  To reach the private
// static members without editing the reference, this translation unit makes
// `private` expand to `public` while it includes the engine header (the
// standard headers are included first, unaffected).
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
using Engine = R::SoftwareComputeEngine;

extern "C" {

// prim: mass, spin, disk inner scale, disk outer (mass units); bodies: n x 11
// (position[3], mass, spin_parameter, axis[3], disk_enabled, inner_scale,
// outer_units).  Outputs: the source table (count x 20: position[3], mass,
// axis[3], spin, frame_x[3], r_+, frame_y[3], sqrt(r_+^2 + a^2), disk inner,
// disk outer), the RHS at (x, p), the initial momentum for `outward` at x, and
// the inside-horizon answer at x.  Returns the source count.
uint32_t ref_ms_case(const double prim[4], uint32_t n, const double* bodies, const double x[3], const double p[3],
                     const double outward[3], double* table, double rhs[6], double p0[3], int* inside) {
	R::GpuCameraPushConstants pc{};
	pc.metric_type = 3;
	pc.metric_mass = prim[0];
	pc.metric_spin = prim[1];
	pc.primary_disk.enabled = 1.0f;
	pc.primary_disk.inner_radius_scale = static_cast<float>(prim[2]);
	pc.primary_disk.outer_radius_mass_units = static_cast<float>(prim[3]);
	pc.hydro_disk.model = 1;
	std::vector<R::GpuBodyData> bs(n);
	for (uint32_t b = 0; b < n; ++b) {
		const double* s = bodies + 11 * b;
		bs[b].preset_3d = 8;
		bs[b].position = {s[0], s[1], s[2], 0.0};
		bs[b].mass = s[3];
		bs[b].spin_parameter = s[4];
		bs[b].spin_axis = {s[5], s[6], s[7], 0.0};
		bs[b].disk.enabled = static_cast<float>(s[8]);
		bs[b].disk.inner_radius_scale = static_cast<float>(s[9]);
		bs[b].disk.outer_radius_mass_units = static_cast<float>(s[10]);
	}
	const auto ms = Engine::build_multi_source_data(pc, std::span<const R::GpuBodyData>(bs.data(), bs.size()));
	for (size_t i = 0; i < ms.count; ++i) {
		double* t = table + 20 * i;
		for (int k = 0; k < 4; ++k) {
			t[k] = ms.position_mass[i][k];
			t[4 + k] = ms.axis_spin[i][k];
			t[8 + k] = ms.frame_x_horizon[i][k];
			t[12 + k] = ms.frame_y_equatorial[i][k];
		}
		t[16] = ms.disk_range[i][0];
		t[17] = ms.disk_range[i][1];
		t[18] = t[19] = 0.0;
	}
	std::array<double, 3> dx{}, dp{};
	Engine::ms_rhs(ms, {x[0], x[1], x[2]}, {p[0], p[1], p[2]}, dx, dp);
	for (int k = 0; k < 3; ++k) {
		rhs[k] = dx[k];
		rhs[3 + k] = dp[k];
	}
	const auto mom = Engine::ms_initial_momentum(ms, {x[0], x[1], x[2]}, {outward[0], outward[1], outward[2]});
	for (int k = 0; k < 3; ++k) p0[k] = mom[k];
	*inside = Engine::ms_inside_horizon(ms, {x[0], x[1], x[2]}) ? 1 : 0;
	return static_cast<uint32_t>(ms.count);
}

}  // extern "C"
