// rt_sky_profile.h -- the procedural sky's settings in the byte layout of the
// reference's GpuSkyProfile (render/gpu_types.hpp:273-964, 1808 bytes), so a
// GpuSkyProfile copies in as it stands.  One list (RT_SKY_FIELDS) gives every
// field in layout order with its type and its default; it defines the struct,
// its defaults and the by-name table of the C ABI (rt_sky_profile_set/get).
#pragma once

#include <cstddef>
#include <cstdint>

namespace relsim {

// X(type, name, default): scalars in layout order.
#define RT_SKY_U32_FIELDS(X)                                                                                     \
    X(uint32_t, enabled, 1u) X(uint32_t, seed, 56u) X(uint32_t, stars_enabled, 1u)                             \
    X(uint32_t, star_profile_model, 0u) X(uint32_t, star_placement_model, 3u)                                  \
    X(uint32_t, star_size_distribution, 1u) X(uint32_t, star_luminosity_distribution, 1u)                      \
    X(uint32_t, star_spike_count, 4u) X(uint32_t, nebula_enabled, 1u) X(uint32_t, nebula_octaves, 5u)           \
    X(uint32_t, nebula_layer_count, 3u) X(uint32_t, clusters_enabled, 0u) X(uint32_t, cluster_placement_model, 0u) \
    X(uint32_t, cluster_size_distribution, 2u) X(uint32_t, cluster_stars_enabled, 1u)                          \
    X(uint32_t, cluster_member_count, 48u) X(uint32_t, cluster_star_profile_model, 0u)                         \
    X(uint32_t, cluster_inherit_star_profile, 1u) X(uint32_t, dust_enabled, 1u) X(uint32_t, dust_fractal_octaves, 5u) \
    X(uint32_t, galaxies_enabled, 1u) X(uint32_t, galaxy_size_distribution, 1u)                                \
    X(uint32_t, galaxy_morphology_model, 0u) X(uint32_t, quasar_enabled, 1u) X(uint32_t, pulsar_enabled, 1u)    \
    X(uint32_t, snr_enabled, 1u) X(uint32_t, grid_enabled, 0u) X(uint32_t, grid_cell_fill_mode, 0u)             \
    X(uint32_t, grid_cell_color_count, 2u) X(uint32_t, grid_subdivisions, 1u) X(uint32_t, grid_show_polar_caps, 0u) \
    X(uint32_t, grid_show_equator, 0u) X(uint32_t, grid_show_meridians, 0u) X(uint32_t, grid_show_ticks, 0u)    \
    X(uint32_t, dynamic_motion, 0u) X(uint32_t, dynamic_rotation, 0u) X(uint32_t, adaptive_fov_quality, 1u)     \
    X(uint32_t, max_star_octaves, 7u) X(uint32_t, pad_u0, 0u) X(uint32_t, pad_u1, 0u)

#define RT_SKY_F64_FIELDS(X)                                                                                     \
    X(double, master_intensity, 1.0) X(double, quality_factor, 1.0) X(double, star_quality_factor, 1.0)         \
    X(double, nebula_quality_factor, 1.0) X(double, cluster_quality_factor, 1.0)                               \
    X(double, dust_quality_factor, 1.0) X(double, quasar_quality_factor, 1.0) X(double, pulsar_quality_factor, 1.0) \
    X(double, snr_quality_factor, 1.0) X(double, adaptive_fov_reference, 90.0)                                 \
    X(double, adaptive_fov_sensitivity, 2.0) X(double, time_seconds, 0.0) X(double, motion_speed, 0.05)        \
    X(double, rotation_rate_deg_s, 0.01)                                                                        \
    X(double, star_density, 91.064) X(double, star_brightness, 1.81) X(double, star_size_scale, 1.0)           \
    X(double, star_size_min, 5e-05) X(double, star_size_max, 0.00263027) X(double, star_size_param, 3.96)      \
    X(double, star_luminosity_param, 1.84) X(double, star_color_variation, 1.0)                                \
    X(double, star_temperature_bias, 0.32) X(double, star_brightness_variation, 0.5)                           \
    X(double, star_scintillation, 0.0) X(double, star_magnitude_limit, 21.0)                                   \
    X(double, star_profile_param, 2.5) X(double, star_profile_param2, 1.0) X(double, star_spike_length, 4.0)   \
    X(double, star_spike_intensity, 0.6) X(double, star_spike_angle_deg, 45.0)                                 \
    X(double, star_profile_softness, 0.15) X(double, star_dirac_concentration, 0.95)                           \
    X(double, star_bloom_radius, 3.0) X(double, star_bloom_intensity, 0.5)                                     \
    X(double, star_galactic_concentration, 2.5)                                                                 \
    X(double, nebula_intensity, 0.23) X(double, nebula_roughness, 0.76) X(double, nebula_frequency, 2.82)      \
    X(double, nebula_plane_thickness, 0.174) X(double, nebula_plane_falloff, 4.09)                             \
    X(double, nebula_asymmetry, 0.43) X(double, nebula_absorption_density, 1.35)                               \
    X(double, nebula_layer_spread, 0.69) X(double, nebula_core_glow, 0.78) X(double, nebula_curl_strength, 0.46) \
    X(double, nebula_color_separation, 1.6) X(double, nebula_ionization_glow, 0.85)                            \
    X(double, nebula_gas_contrast, 1.94)                                                                        \
    X(double, cluster_density, 0.184) X(double, cluster_brightness, 0.0) X(double, cluster_size_scale, 1.61)   \
    X(double, cluster_size_min, 0.001) X(double, cluster_size_max, 0.0488) X(double, cluster_concentration, 3.76) \
    X(double, cluster_star_density_boost, 2.0) X(double, cluster_halo_radius, 0.27)                            \
    X(double, cluster_plane_scale_height, 0.15) X(double, cluster_member_size, 0.0006)                         \
    X(double, cluster_member_brightness, 1.2) X(double, cluster_halo_intensity, 0.04)                          \
    X(double, cluster_spread_factor, 4.4)                                                                       \
    X(double, dust_density, 3.85) X(double, dust_intensity, 1.3) X(double, dust_scale, 3.82)                   \
    X(double, dust_absorption_ratio, 0.8) X(double, dust_contrast, 3.54)                                       \
    X(double, galaxy_density, 0.5) X(double, galaxy_brightness, 0.07) X(double, galaxy_size_scale, 1.0)        \
    X(double, galaxy_size_min, 0.0005) X(double, galaxy_size_max, 0.0302) X(double, galaxy_size_param, 1.5)    \
    X(double, galaxy_spiral_arms, 5.0) X(double, galaxy_pitch_angle, 1.46) X(double, galaxy_core_ratio, 0.52)  \
    X(double, galaxy_ellipticity_variance, 0.93) X(double, galaxy_bar_strength, 1.07)                          \
    X(double, galaxy_dust_lane_opacity, 0.37) X(double, galaxy_clumpiness, 0.69)                               \
    X(double, galaxy_disk_thickness, 0.19) X(double, galaxy_inclination_variance, 0.89)                        \
    X(double, galaxy_bulge_sersic_index, 3.72) X(double, galaxy_weight_grand_design, 1.55)                     \
    X(double, galaxy_weight_flocculent, 2.5) X(double, galaxy_weight_barred, 0.5)                              \
    X(double, galaxy_weight_elliptical, 0.41) X(double, galaxy_weight_lenticular, 1.21)                        \
    X(double, galaxy_weight_ring, 0.19)                                                                         \
    X(double, quasar_density, 1.136) X(double, quasar_brightness, 1.2) X(double, quasar_core_size, 0.0003)     \
    X(double, quasar_jet_length, 0.08) X(double, quasar_jet_intensity, 1.5)                                    \
    X(double, quasar_jet_opening_angle_deg, 5.0) X(double, quasar_jet_lorentz_factor, 3.06)                    \
    X(double, quasar_accretion_disk_glow, 1.21) X(double, quasar_precession_angle_deg, 11.7)                   \
    X(double, pulsar_density, 0.01) X(double, pulsar_brightness, 1.0) X(double, pulsar_pulse_rate, 2.5)        \
    X(double, pulsar_pulse_duty, 0.15) X(double, pulsar_beam_width_deg, 8.0)                                   \
    X(double, pulsar_magnetic_tilt_deg, 30.0) X(double, pulsar_wind_nebula_scale, 0.0062)                      \
    X(double, pulsar_wind_nebula_intensity, 0.22) X(double, pulsar_frequency_spread, 0.75)                     \
    X(double, snr_density, 0.06) X(double, snr_brightness, 1.2) X(double, snr_shell_thickness, 0.08)           \
    X(double, snr_expansion_age, 0.34) X(double, snr_size, 0.0044) X(double, snr_asymmetry, 0.4)               \
    X(double, snr_filament_scale, 6.13) X(double, snr_interior_glow, 0.07) X(double, snr_color_variation, 1.87) \
    X(double, snr_morphology_variety, 0.6)                                                                      \
    X(double, grid_opacity, 0.5) X(double, grid_line_width, 0.0001) X(double, grid_spacing_deg, 30.0)          \
    X(double, grid_glow, 0.0) X(double, grid_tick_interval_deg, 5.0) X(double, grid_tick_length, 0.003)        \
    X(double, grid_tick_width, 0.0001) X(double, grid_cell_opacity, 0.1) X(double, grid_equator_width, 0.007)  \
    X(double, grid_equator_opacity, 0.8) X(double, grid_polar_width, 0.003) X(double, grid_polar_opacity, 0.7) \
    X(double, grid_meridian_width, 0.003) X(double, grid_meridian_opacity, 0.7)                                \
    X(double, grid_major_width, 0.005) X(double, grid_minor_width, 0.003)                                      \
    X(double, hue_shift_deg, 0.0) X(double, saturation, 0.84) X(double, orientation_yaw_deg, 0.0)              \
    X(double, orientation_pitch_deg, 0.0) X(double, orientation_roll_deg, 0.0)                                 \
    X(double, grid_orientation_yaw_deg, 0.0) X(double, grid_orientation_pitch_deg, 0.0)                        \
    X(double, grid_orientation_roll_deg, 0.0) X(double, pad_d0, 0.0)

// X(name, a, b, c): three floats and a pad float each.
#define RT_SKY_VEC_FIELDS(X)                                                                                     \
    X(nebula_plane_normal, 0.0f, 0.4472136f, 0.8944272f) X(nebula_asymmetry_dir, 0.7071068f, 0.0f, 0.7071068f)  \
    X(nebula_emission_color, 0.92f, 0.22f, 0.38f) X(nebula_secondary_color, 0.15f, 0.72f, 0.90f)                \
    X(nebula_tertiary_color, 0.95f, 0.65f, 0.15f) X(cluster_core_tint, 1.1f, 1.0f, 0.8f)                        \
    X(dust_tint, 0.4f, 0.25f, 0.15f) X(grid_major_color, 1.0f, 1.0f, 1.0f)                                      \
    X(grid_minor_color, 0.470588f, 0.470588f, 0.470588f) X(background_color, 0.0f, 0.0f, 0.0f)                  \
    X(grid_equator_color, 0.95f, 0.30f, 0.30f) X(grid_polar_color, 0.298039f, 0.952941f, 0.298039f)              \
    X(grid_meridian_color, 0.298039f, 0.298039f, 0.952941f) X(grid_tick_color, 1.0f, 1.0f, 1.0f)                 \
    X(snr_shell_color, 1.35f, 0.65f, 0.45f) X(snr_interior_color, 0.35f, 0.70f, 1.25f)

struct SkyProfile {
#define RT_SKY_DECL(T, N, D) T N = D;
    RT_SKY_U32_FIELDS(RT_SKY_DECL)
    RT_SKY_F64_FIELDS(RT_SKY_DECL)
#undef RT_SKY_DECL
#define RT_SKY_VDECL(N, A, B, C) float N[4] = {A, B, C, 0.0f};
    RT_SKY_VEC_FIELDS(RT_SKY_VDECL)
#undef RT_SKY_VDECL
    float grid_cell_colors[16][4] = {{0.10f, 0.12f, 0.18f, 0.0f}, {0.05f, 0.07f, 0.12f, 0.0f},
                                     {0.08f, 0.15f, 0.15f, 0.0f}, {0.15f, 0.10f, 0.12f, 0.0f},
                                     {0.14f, 0.14f, 0.08f, 0.0f}, {0.12f, 0.06f, 0.14f, 0.0f},
                                     {0.06f, 0.12f, 0.14f, 0.0f}, {0.14f, 0.08f, 0.06f, 0.0f},
                                     {0.08f, 0.10f, 0.16f, 0.0f}, {0.16f, 0.08f, 0.10f, 0.0f},
                                     {0.10f, 0.16f, 0.08f, 0.0f}, {0.08f, 0.16f, 0.16f, 0.0f},
                                     {0.16f, 0.16f, 0.08f, 0.0f}, {0.16f, 0.08f, 0.16f, 0.0f},
                                     {0.12f, 0.12f, 0.12f, 0.0f}, {0.06f, 0.06f, 0.06f, 0.0f}};
};
static_assert(sizeof(SkyProfile) == 1808, "GpuSkyProfile layout");

}  // namespace relsim
