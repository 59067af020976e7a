// relsim_executor.hpp -- C++ adapter with the method names and semantics of
// Render::VulkanComputeExecutor (include/relativistic/render/vulkan_compute_executor.hpp:29)
// over the tracer's C ABI (relsim_cuda.h).  Header only; link librelsim_cuda.so.
//
//   reference                                        here
//   initialize(VulkanContext&)            :983       initialize(int device)
//   is_ready() const                      :1257      is_ready()
//   shutdown()                            :1272      shutdown()
//   dispatch_and_readback(params, out, bodies, cancel)  :1399-1464
//                                                    dispatch_and_readback(camera, out, cancel)
//   dispatch_tile_and_readback(params, out, bodies)     :1372-1391
//                                                    dispatch_tile_and_readback(camera, out)
//   static is_platform_supported()        :1634      is_platform_supported()
//
// Semantics kept from the reference: bool returns and no exceptions across the
// boundary; the output vector is resized by the callee (row window x width, or
// tile extent); the cancel flag is polled between bands and a cancelled
// dispatch returns false; a device error clears is_ready(), after which the
// caller falls back as GeodesicComputePipeline does
// (geodesic_compute_pipeline.hpp:508-524).  Calls on one executor are
// serialised by the caller (gpu_mutex_ in the reference).  Scene bodies are not
// part of this path (the pipeline's eligibility gate sends body scenes
// elsewhere).
#ifndef RELSIM_EXECUTOR_HPP
#define RELSIM_EXECUTOR_HPP

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "relsim_cuda.h"

namespace relsim {

// Integration settings of the tracer that GpuCameraPushConstants does not carry.
struct TraceSettings {
    double rtol = 1e-10;
    double atol = 1e-10;
    double capture_scale = 1.01;    // captured when r_BL < capture_scale * r_+
    uint32_t precision = RT_PRECISION_FP64;
    uint32_t early_capture = 1;
};

// Metric types of GpuCameraPushConstants this backend traces
// (trace_exact_photon_dispatch, software_compute_engine.hpp:3316-3392):
// 2 and 3 Kerr-Schild Kerr; 5 Kerr-Newman and 1 Schwarzschild in
// Boyer-Lindquist coordinates.
inline bool metric_type_supported(uint32_t metric_type) {
    return metric_type == 1u || metric_type == 2u || metric_type == 3u || metric_type == 5u;
}

// rt_camera from the reference's push constants (gpu_types.hpp:966-1109): the
// observer, tetrad, field of view, metric (type, mass, spin, charge), escape
// radius, image size, step budget, row window and tile, and the primary disk
// (inner = inner_radius_scale x r_ISCO(a), outer = outer_radius_mass_units x M).
// A template so that this header does not depend on the reference's headers.
template <class PushConstants>
rt_camera camera_from_push_constants(const PushConstants& p, const TraceSettings& s = {}) {
    rt_camera c;
    rt_camera_defaults(&c);
    for (int i = 0; i < 4; ++i) {
        c.observer_position[i] = p.observer_position[i];
        c.tetrad_e1[i] = p.tetrad_e1[i];
        c.tetrad_e2[i] = p.tetrad_e2[i];
        c.tetrad_e3[i] = p.tetrad_e3[i];
    }
    c.field_of_view_rad = p.field_of_view_rad;
    c.metric_mass = std::max(p.metric_mass, 1e-4);
    c.metric_spin = std::clamp(p.metric_spin, -0.999 * c.metric_mass, 0.999 * c.metric_mass);
    if (p.metric_type == 5u) {  // KerrNewmanMetric (:3364-3368)
        c.metric_form = RT_METRIC_BOYER_LINDQUIST;
        c.metric_charge = p.metric_charge;
    } else if (p.metric_type == 1u) {  // Schwarzschild: spin and charge unused
        c.metric_form = RT_METRIC_BOYER_LINDQUIST;
        c.metric_spin = 0.0;
        c.metric_charge = 0.0;
    }
    c.escape_radius = p.escape_radius;
    c.screen_width = p.screen_width;
    c.screen_height = p.screen_height;
    c.max_integration_steps = p.max_integration_steps;
    c.dispatch_row_offset = p.dispatch_row_offset;
    c.dispatch_row_count = p.dispatch_row_count;
    c.tile_origin_x = p.tile_origin_x;
    c.tile_origin_y = p.tile_origin_y;
    c.tile_extent_x = p.tile_extent_x;
    c.tile_extent_y = p.tile_extent_y;
    const double scale = static_cast<double>(p.primary_disk.inner_radius_scale);
    c.disk_inner_radius = (scale == 1.0) ? 0.0 : scale * rt_kerr_isco_radius(c.metric_mass, c.metric_spin);
    c.disk_outer_radius = static_cast<double>(p.primary_disk.outer_radius_mass_units) * c.metric_mass;
    c.rtol = s.rtol;
    c.atol = s.atol;
    c.capture_scale = s.capture_scale;
    c.precision_mode = s.precision;
    c.early_capture = s.early_capture;
    return c;
}

// rt_shading from the reference's push constants: primary_disk (a
// GpuDiskProfile, copied as it lies), the disk temperature, saturation and
// beaming overrides, time, exposure, tonemapping mode, the hydro disk model
// with its accretion rate and torus settings, and the procedural sky (params.sky, a
// GpuSkyProfile copied as it lies).  The reference's image panoramas
// (sky_background_source != 0) are not part of the library: such a scene
// keeps the procedural sky.
template <class PushConstants>
rt_shading shading_from_push_constants(const PushConstants& p) {
    rt_shading s;
    rt_shading_defaults(&s);
    static_assert(sizeof(p.primary_disk) == sizeof(rt_disk_profile), "GpuDiskProfile layout");
    std::memcpy(&s.disk, &p.primary_disk, sizeof s.disk);
    s.disk_temperature_scale_k = p.disk_temperature_scale_k;
    s.disk_temperature_floor_k = p.disk_temperature_floor_k;
    s.disk_color_saturation = p.disk_color_saturation;
    s.disk_doppler_beaming_exponent = p.disk_doppler_beaming_exponent;
    s.time = p.time;
    s.camera_exposure = p.camera_exposure;
    s.tonemapping_mode = p.tonemapping_mode;
    s.hydro_model = p.hydro_disk.model;
    s.accretion_rate_scale = p.hydro_disk.accretion_rate_scale;
    s.torus_inner_radius = p.hydro_disk.torus_inner_radius;
    s.torus_center_radius = p.hydro_disk.torus_center_radius;
    s.adiabatic_index = p.hydro_disk.adiabatic_index;
    s.optical_depth_scale = p.hydro_disk.optical_depth_scale;
    s.sampling_density = p.hydro_disk.sampling_density;
    static_assert(sizeof(p.sky) == sizeof(rt_sky_profile), "GpuSkyProfile layout");
    std::memcpy(&s.sky, &p.sky, sizeof s.sky);
    s.sky_enabled = 1;
    return s;
}

class CudaComputeExecutor {
public:
    CudaComputeExecutor() = default;
    CudaComputeExecutor(const CudaComputeExecutor&) = delete;
    CudaComputeExecutor& operator=(const CudaComputeExecutor&) = delete;
    ~CudaComputeExecutor() { shutdown(); }

    [[nodiscard]] static bool is_platform_supported() { return rt_is_platform_supported() != 0; }

    [[nodiscard]] bool initialize(int device = 0) {
        shutdown();
        const rt_status st = rt_create(&h_, device);
        if (st != RT_OK) {
            error_ = "rt_create failed (no sm_100 device?)";
            h_ = nullptr;
            return false;
        }
        return true;
    }

    [[nodiscard]] bool is_ready() const noexcept { return h_ != nullptr && rt_is_ready(h_) != 0; }

    // Shade the pixels of later dispatches (nullptr: colour off, the default).
    [[nodiscard]] bool set_shading(const rt_shading* s) { return h_ != nullptr && check(rt_set_shading(h_, s)); }

    void shutdown() noexcept {
        if (h_) rt_destroy(h_);
        h_ = nullptr;
    }

    const std::string& last_error() const noexcept { return error_; }
    rt_handle* handle() noexcept { return h_; }

    // Row window of the image, banded so that `cancel` is polled between bands.
    // Pixel: rt_pixel_out or any 32-byte standard-layout type of the same layout
    // (the reference's GpuPixelOutput).
    template <class Pixel = rt_pixel_out>
    [[nodiscard]] bool dispatch_and_readback(const rt_camera& camera, std::vector<Pixel>& output,
                                             const std::atomic<bool>* cancel = nullptr,
                                             const rt_ray_out* rays = nullptr) {
        static_assert(sizeof(Pixel) == sizeof(rt_pixel_out) && std::is_standard_layout_v<Pixel>,
                      "pixel type must have the 32-byte GpuPixelOutput layout");
        if (!is_ready() || camera.screen_width == 0 || camera.screen_height == 0) return false;
        const uint32_t first = std::min(camera.dispatch_row_offset, camera.screen_height);
        const uint32_t rows = (camera.dispatch_row_count == 0)
                                  ? camera.screen_height - first
                                  : std::min(camera.dispatch_row_count, camera.screen_height - first);
        if (rows == 0) return false;
        const size_t width = camera.screen_width;
        if (output.size() != width * rows) output.resize(width * rows);
        const uint32_t band = static_cast<uint32_t>(std::max<size_t>(1, kBandRays / width));
        for (uint32_t r = 0; r < rows; r += band) {
            if (cancel && cancel->load(std::memory_order_relaxed)) return false;
            rt_camera c = camera;
            c.dispatch_row_offset = first + r;
            c.dispatch_row_count = std::min(band, rows - r);
            const size_t offset = static_cast<size_t>(r) * width;
            rt_ray_out part{};
            if (rays) part = offset_rays(*rays, offset);
            if (!check(rt_dispatch(h_, &c, reinterpret_cast<rt_pixel_out*>(output.data() + offset),
                                   rays ? &part : nullptr,
                                   width * c.dispatch_row_count, nullptr)))
                return false;
        }
        return true;
    }

    // Tile [origin, origin + extent), tile-major; output resized to the extent.
    template <class Pixel = rt_pixel_out>
    [[nodiscard]] bool dispatch_tile_and_readback(const rt_camera& camera, std::vector<Pixel>& output) {
        static_assert(sizeof(Pixel) == sizeof(rt_pixel_out) && std::is_standard_layout_v<Pixel>,
                      "pixel type must have the 32-byte GpuPixelOutput layout");
        if (!is_ready() || camera.tile_extent_x == 0 || camera.tile_extent_y == 0) return false;
        if (camera.tile_origin_x >= camera.screen_width || camera.tile_origin_y >= camera.screen_height) return false;
        const size_t n = static_cast<size_t>(camera.tile_extent_x) * camera.tile_extent_y;
        if (output.size() != n) output.resize(n);
        return check(rt_dispatch_tile(h_, &camera, reinterpret_cast<rt_pixel_out*>(output.data()), nullptr, n));
    }

private:
    static constexpr size_t kBandRays = size_t{1} << 22;

    static rt_ray_out offset_rays(const rt_ray_out& r, size_t k) {
        rt_ray_out o = r;
        auto adv = [k](auto*& p) {
            if (p) p += k;
        };
        adv(o.status), adv(o.flags), adv(o.steps_accepted), adv(o.steps_rejected);
        adv(o.r), adv(o.theta), adv(o.phi), adv(o.r_hit), adv(o.g), adv(o.lambda);
        adv(o.dH), adv(o.dE), adv(o.dLz), adv(o.dQ);
        adv(o.exit_x), adv(o.exit_y), adv(o.exit_z), adv(o.body);
        return o;
    }

    bool check(rt_status st) {
        if (st == RT_OK) return true;
        error_ = rt_last_error(h_);
        return false;
    }

    rt_handle* h_ = nullptr;
    std::string error_;
};

}  // namespace relsim

#endif
