// Host-side code under AddressSanitizer and UndefinedBehaviorSanitizer: the
// library's per-camera table builders (csrc/rt_bundle.cpp: Kerr-Schild bundle,
// Boyer-Lindquist bundle, multi-source source table and bundle, ISCO, horizon,
// row windows) over cameras at and beyond their clamps, and the CPU oracles
// (Kerr-Schild, multi-source, Boyer-Lindquist traces of a few rays, shading).
// Built and run by tests/test_host_sanitizers.py; exits 0 and prints "ok".
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ks_oracle.h"
#include "rt_internal.h"

using namespace relsim;

namespace {

constexpr double kPi = 3.14159265358979323846;

rt_camera camera(double spin, double r_obs, double incl_deg, double fov_deg, uint32_t w, uint32_t h) {
    rt_camera c;
    std::memset(&c, 0, sizeof c);
    c.field_of_view_rad = fov_deg * kPi / 180.0;
    c.metric_mass = 1.0;
    c.metric_spin = spin;
    c.escape_radius = 1000.0;
    c.capture_scale = 1.01;
    c.disk_outer_radius = 20.0;
    c.rtol = c.atol = 1e-8;
    c.step_cap_fraction = 0.1;
    c.initial_step_fraction = 0.01;
    c.projection_tol = 1e-12;
    c.screen_width = w;
    c.screen_height = h;
    c.max_integration_steps = 3000;
    c.early_capture = 1;
    const double th = incl_deg * kPi / 180.0, st = std::sin(th), ct = std::cos(th);
    c.observer_position[1] = r_obs;
    c.observer_position[2] = th;
    const double er[3] = {st, 0.0, ct}, eth[3] = {ct, 0.0, -st}, eph[3] = {0.0, 1.0, 0.0};
    for (int i = 0; i < 3; ++i) {
        c.tetrad_e1[1 + i] = -er[i];
        c.tetrad_e2[1 + i] = eph[i];
        c.tetrad_e3[1 + i] = -eth[i];
    }
    return c;
}

orc_camera to_orc(const rt_camera& c) {
    orc_camera o;
    std::memset(&o, 0, sizeof o);
    std::memcpy(o.observer_position, c.observer_position, sizeof o.observer_position);
    std::memcpy(o.tetrad_e1, c.tetrad_e1, sizeof o.tetrad_e1);
    std::memcpy(o.tetrad_e2, c.tetrad_e2, sizeof o.tetrad_e2);
    std::memcpy(o.tetrad_e3, c.tetrad_e3, sizeof o.tetrad_e3);
    o.field_of_view_rad = c.field_of_view_rad;
    o.metric_mass = c.metric_mass;
    o.metric_spin = c.metric_spin;
    o.escape_radius = c.escape_radius;
    o.capture_scale = c.capture_scale;
    o.disk_inner_radius = c.disk_inner_radius;
    o.disk_outer_radius = c.disk_outer_radius;
    o.rtol = c.rtol;
    o.atol = c.atol;
    o.step_cap_fraction = c.step_cap_fraction;
    o.initial_step_fraction = c.initial_step_fraction;
    o.projection_tol = c.projection_tol;
    o.screen_width = c.screen_width;
    o.screen_height = c.screen_height;
    o.max_steps = c.max_integration_steps;
    o.early_capture = c.early_capture;
    return o;
}

int failures = 0;

void expect(bool ok, const char* what) {
    if (!ok) {
        std::printf("FAILED: %s\n", what);
        ++failures;
    }
}

}  // namespace

int main() {
    // cameras at and beyond their clamps: spin past 0.999 M, negative spin,
    // an observer inside 1.02 r_+, one-pixel and ragged screens, row windows
    const rt_camera cams[] = {camera(0.94, 100.0, 17.0, 12.0, 64, 48),  camera(0.99995, 60.0, 80.0, 20.0, 1, 1),
                              camera(-0.97, 30.0, 120.0, 30.0, 37, 5), camera(0.5, 1.5, 60.0, 60.0, 3, 100),
                              camera(0.0, 50.0, 60.0, 30.0, 33, 31)};
    for (const rt_camera& c0 : cams) {
        rt_camera c = c0;
        for (uint32_t off : {0u, 1u, c.screen_height - 1, c.screen_height + 5}) {
            c.dispatch_row_offset = off;
            c.dispatch_row_count = 2;
            uint32_t row0 = 0, nrows = 0;
            row_window(c, row0, nrows);
            expect(row0 + nrows <= c.screen_height, "row window inside the screen");
        }
        c.dispatch_row_offset = c.dispatch_row_count = 0;
        BundleDesc b;
        build_bundle(c, 0, c.screen_width, 0, c.screen_height, 0, 0, b);
        expect(std::isfinite(b.h0) && b.h0 > 0.0, "bundle step");
        expect(kerr_isco_radius(1.0, c.metric_spin) > 0.0, "isco");
        rt_camera bl = c;
        bl.metric_form = RT_METRIC_BOYER_LINDQUIST;
        bl.metric_charge = 0.2;
        if (std::fabs(bl.metric_spin) < 0.9) {
            BlDesc d;
            build_bl_bundle(bl, 0, bl.screen_width, 0, bl.screen_height, 0, 0, d);
            expect(kn_horizon(1.0, bl.metric_spin, 0.2) > 1.0, "Kerr-Newman horizon");
        }
        // multi-source tables: no bodies, and the largest (15 bodies)
        std::vector<rt_source> src(15);
        for (uint32_t i = 0; i < src.size(); ++i) {
            std::memset(&src[i], 0, sizeof src[i]);
            src[i].position[0] = 10.0 + 2.0 * i;
            src[i].position[1] = -5.0 + i;
            src[i].position[2] = 3.0 - 0.5 * i;
            src[i].mass = 0.2 + 0.05 * i;
            src[i].spin_parameter = (i % 3 == 0) ? 1.5 : 0.3;  // beyond the clamp on some
            src[i].axis[0] = (i % 2) ? 0.0 : 1.0;               // a zero axis on others
            src[i].disk_enabled = 1.0;
            src[i].disk_outer_units = 10.0;
        }
        MsSource table[kMaxSources];
        for (uint32_t n : {0u, 1u, 15u}) {
            const uint32_t count = build_ms_sources(c, src.data(), n, table);
            expect(count == n + 1, "source count");
            MsDesc md;
            build_ms_bundle(c, 0, c.screen_width, 0, c.screen_height, 0, 0, 0, count, md);
        }
    }

    // the oracles: a few rays of each tracer form
    const rt_camera c = camera(0.9, 40.0, 70.0, 30.0, 24, 24);
    const orc_camera oc = to_orc(c);
    std::vector<orc_ray> rays(24);
    orc_trace(&oc, nullptr, 12 * 24, 24, rays.data(), 2);
    for (const orc_ray& r : rays) expect(r.status <= 3, "ks class");
    orc_bl_trace(&oc, 0.3, nullptr, 12 * 24, 24, rays.data(), 2);
    for (const orc_ray& r : rays) expect(r.status <= 3, "bl class");
    orc_source os[3];
    std::memset(os, 0, sizeof os);
    for (int i = 0; i < 3; ++i) {
        os[i].position[0] = 12.0 + 4.0 * i;
        os[i].position[1] = 6.0 - 3.0 * i;
        os[i].mass = 0.5;
        os[i].spin_parameter = 0.5;
        os[i].axis[2] = 1.0;
        os[i].disk_enabled = 1.0;
        os[i].disk_outer_units = 12.0;
    }
    orc_ms_table t;
    orc_ms_build(&oc, os, 3, &t);
    orc_ms_trace(&oc, &t, nullptr, 12 * 24, 24, rays.data(), 2);
    for (const orc_ray& r : rays) expect(r.status <= 3, "ms class");
    float profile[32] = {}, resolved[32];
    const double over[4] = {0.0, 0.0, 0.0, 0.0};
    orc_resolve_profile(profile, over, resolved);
    float px[3];
    for (uint32_t mode = 0; mode < 4; ++mode) {
        orc_shade_pixel(resolved, mode % 2, 1.0f, mode, 0.0, 1.0, 0.9, 2.32, 20.0, 0.0, 0.5, 3, 7.5, 1.0, 0.8, px);
        expect(std::isfinite(px[0]) && std::isfinite(px[1]) && std::isfinite(px[2]), "shaded pixel");
    }
    if (failures) return 1;
    std::printf("ok\n");
    return 0;
}
