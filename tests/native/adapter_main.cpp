// Drives relsim::CudaComputeExecutor (include/relsim_executor.hpp) the way the
// reference's pipeline drives VulkanComputeExecutor.  Used by tests/test_adapter.py.
//   adapter_main map                 print the mapped camera of a push-constant struct
//   adapter_main route               metric type routing: form, spin, charge for types 3, 5, 1
//   adapter_main shade               the push constants' shading settings as rt_shading
//   adapter_main cpu                 platform/initialise answers without a device
//   adapter_main gpu <out.bin>       dispatch_and_readback of a 96x64 image -> raw pixels; cancel check
#include <atomic>
#include <cstdio>
#include <cstring>
#include <vector>

#ifdef RELSIM_WITH_REFERENCE_TYPES
#include "relativistic/render/gpu_types.hpp"
using Push = Relativistic::Render::GpuCameraPushConstants;
#else
#include <array>
struct DiskProfile {  // GpuDiskProfile's 32 floats (gpu_types.hpp:42-75)
    float enabled = 1.0f, inner_radius_scale = 1.0f, outer_radius_mass_units = 24.0f, peak_temperature_k = 9500.0f;
    float floor_temperature_k = 1200.0f, temperature_exponent = 0.75f, zero_torque_strength = 1.0f;
    float extra_beaming_exponent = 2.0f, brightness = 0.45f, color_saturation = 1.0f, tint_strength = 0.0f;
    float opacity_scale = 1.0f, tint_r = 1.0f, tint_g = 1.0f, tint_b = 1.0f, rotation_speed_scale = 4.0f;
    float ring_amplitude = 0.35f, ring_frequency = 9.0f, ring_sharpness = 3.0f, spiral_arm_count = 2.0f;
    float spiral_pitch = 1.2f, spiral_amplitude = 0.25f, turbulence_amplitude = 0.45f, turbulence_scale = 5.0f;
    float turbulence_octaves = 4.0f, radial_stretch = 3.0f, grain_amplitude = 0.2f, grain_scale = 40.0f;
    float reference_luminance = 1.0f, noise_seed = 1.0f, temperature_normalization = 1.0f, edge_softness = 1.0f;
};
struct HydroDisk {
    uint32_t model = 0;
    float accretion_rate_scale = 1.0f;
    float torus_inner_radius = 6.0f, torus_center_radius = 12.0f, adiabatic_index = 1.3333334f;
    float optical_depth_scale = 0.35f, sampling_density = 2.0f;
};
struct Push {  // the fields of GpuCameraPushConstants the tracer reads (gpu_types.hpp:966-1109)
    std::array<double, 4> observer_position{}, tetrad_e1{}, tetrad_e2{}, tetrad_e3{};
    double field_of_view_rad = 1.0471975511965976, metric_mass = 1.0, metric_spin = 0.0, escape_radius = 100.0;
    double metric_charge = 0.0;
    uint32_t metric_type = 3;
    double time = 0.0, camera_exposure = 0.0;
    double disk_temperature_scale_k = 23796.0, disk_temperature_floor_k = 1200.0;
    double disk_doppler_beaming_exponent = 5.32, disk_color_saturation = 1.0;
    uint32_t tonemapping_mode = 0;
    HydroDisk hydro_disk{};
    uint32_t screen_width = 3840, screen_height = 2160, max_integration_steps = 2048;
    uint32_t dispatch_row_offset = 0, dispatch_row_count = 0;
    uint32_t tile_origin_x = 0, tile_origin_y = 0, tile_extent_x = 0, tile_extent_y = 0;
    DiskProfile primary_disk{};
    struct {
        unsigned char bytes[1808];
    } sky{};  // a GpuSkyProfile image
};
#endif
#include "relsim_executor.hpp"

static Push headline_push(uint32_t w, uint32_t h) {
    rt_camera d;
    rt_camera_defaults(&d);  // r=100, i=17 deg, FOV 12 deg, a=0.94
    Push p{};
    for (int i = 0; i < 4; ++i) {
        p.observer_position[i] = d.observer_position[i];
        p.tetrad_e1[i] = d.tetrad_e1[i];
        p.tetrad_e2[i] = d.tetrad_e2[i];
        p.tetrad_e3[i] = d.tetrad_e3[i];
    }
    p.field_of_view_rad = d.field_of_view_rad;
    p.metric_mass = 1.0;
    p.metric_spin = 0.94;
    p.metric_type = 3;
    p.metric_charge = 0.0;
    p.escape_radius = 1000.0;
    p.screen_width = w;
    p.screen_height = h;
    p.max_integration_steps = 20000;
    p.primary_disk.inner_radius_scale = 1.0f;
    p.primary_disk.outer_radius_mass_units = 20.0f;
    return p;
}

int main(int argc, char** argv) {
    const char* mode = argc > 1 ? argv[1] : "map";
    if (!std::strcmp(mode, "map")) {
        Push p = headline_push(96, 64);
        p.metric_spin = 1.5;  // clamped to 0.999 M
        p.primary_disk.inner_radius_scale = 1.5f;
        const rt_camera c = relsim::camera_from_push_constants(p);
#ifdef RELSIM_WITH_REFERENCE_TYPES
        // the executor takes the reference's own pixel vector (compile-time layout check)
        std::vector<Relativistic::Render::GpuPixelOutput> ref_pixels;
        relsim::CudaComputeExecutor unused;
        if (argc > 99) (void)unused.dispatch_and_readback(c, ref_pixels);
#endif
        std::printf("%.17g %.17g %.17g %.17g %u %u %u %.17g\n", c.metric_spin, c.disk_inner_radius,
                    c.disk_outer_radius, c.escape_radius, c.screen_width, c.screen_height, c.max_integration_steps,
                    rt_kerr_isco_radius(1.0, 0.999));
        return 0;
    }
    if (!std::strcmp(mode, "route")) {
        for (uint32_t type : {3u, 5u, 1u}) {
            Push p = headline_push(32, 32);
            p.metric_type = type;
            p.metric_charge = 0.4;
            const rt_camera c = relsim::camera_from_push_constants(p);
            std::printf("%u %d %u %.17g %.17g\n", type, relsim::metric_type_supported(type) ? 1 : 0, c.metric_form,
                        c.metric_spin, c.metric_charge);
        }
        std::printf("%d %d\n", relsim::metric_type_supported(4u) ? 1 : 0, relsim::metric_type_supported(0u) ? 1 : 0);
        return 0;
    }
    if (!std::strcmp(mode, "shade")) {
        Push p = headline_push(32, 32);
        p.primary_disk.ring_frequency = 7.0f;
        p.disk_temperature_scale_k = 15000.0;
        p.disk_doppler_beaming_exponent = 3.0;
        p.time = 2.5;
        p.camera_exposure = -1.0;
        p.tonemapping_mode = 1;
        p.hydro_disk.model = 1;
        p.hydro_disk.accretion_rate_scale = 2.0f;
        p.hydro_disk.torus_center_radius = 11.0f;
        p.hydro_disk.sampling_density = 3.0f;
        const rt_shading s = relsim::shading_from_push_constants(p);
        std::printf("%g %g %g %g %g %u %u %g %u %g %g %g %g %g %g\n", s.disk.ring_frequency, s.disk_temperature_scale_k,
                    s.disk_doppler_beaming_exponent, s.time, s.camera_exposure, s.tonemapping_mode, s.hydro_model,
                    s.accretion_rate_scale, s.sky_enabled, s.disk.edge_softness, s.torus_inner_radius,
                    s.torus_center_radius, s.adiabatic_index, s.optical_depth_scale, s.sampling_density);
        return 0;
    }
    if (!std::strcmp(mode, "cpu")) {
        relsim::CudaComputeExecutor ex;
        const bool sup = relsim::CudaComputeExecutor::is_platform_supported();
        const bool init = ex.initialize(0);
        std::vector<rt_pixel_out> out;
        const rt_camera c = relsim::camera_from_push_constants(headline_push(32, 32));
        const bool disp = ex.dispatch_and_readback(c, out);
        std::printf("%d %d %d %d\n", sup, init, ex.is_ready(), disp);
        return 0;
    }
    if (!std::strcmp(mode, "gpu") && argc > 2) {
        relsim::CudaComputeExecutor ex;
        if (!ex.initialize(0)) return 2;
        const rt_camera c = relsim::camera_from_push_constants(headline_push(96, 64));
        std::vector<rt_pixel_out> out;
        if (!ex.dispatch_and_readback(c, out)) return 3;
        FILE* f = std::fopen(argv[2], "wb");
        if (!f) return 4;
        std::fwrite(out.data(), sizeof(rt_pixel_out), out.size(), f);
        std::fclose(f);
        std::atomic<bool> cancel{true};
        std::vector<rt_pixel_out> out2;
        const bool cancelled_ok = !ex.dispatch_and_readback(c, out2, &cancel);
        std::printf("%zu %d %d\n", out.size(), cancelled_ok, ex.is_ready());
        return 0;
    }
    return 1;
}
