"""Pixel shading pass (rt_set_shading, csrc/rt_shade.cu) against the shading
oracle (oracle/shade_oracle.c, pinned bit for bit to the reference's
AccretionDiskModel::shade, Novikov-Thorne context, blackbody colour and
apply_tonemapping by tests/test_oracle_shading.py).

Kerr-Schild cameras are shaded as the reference's image path does, through a
translucent disk (software_compute_engine.hpp:1734-1765): each disk crossing
adds its radiance at the throughput left and lowers the throughput by its
opacity, and the ray goes on while more than 0.01 is left.  These pixels are
compared with the oracle's own continuation trace (oracle.trace_cont, every
crossing recorded) shaded by the oracle (orc_shade_cont); the per-ray record
keeps describing the first hit, unchanged by shading.  Boyer-Lindquist
cameras end at the first crossing; there the oracle shades each ray from the
GPU's own record (class, r_hit, phi, g), which isolates the shading
arithmetic: CUDA's float cosf/powf/expf and FMA contraction differ from the
host's in the last bits (bar 1e-6 sRGB, measured 1.8e-7).  Rays that are not
disk hits are exactly black with alpha 1 (the sky is disabled).
"""
import ctypes
import math

import numpy as np
import pytest

import relsim
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CONT_BAR = 1e-5        # FP64 tracer through the translucent disk vs the oracle's continuation (sRGB)
MIXED_CONT_BAR = 1e-4  # mixed tracer through the translucent disk vs the FP64 oracle (sRGB)


def _camera_constants(cam):
    m = max(cam.metric_mass, 1e-4)
    a = min(max(cam.metric_spin, -0.999 * m), 0.999 * m)
    inner = cam.disk_inner_radius if cam.disk_inner_radius > 0 else relsim.lib().rt_kerr_isco_radius(m, a)
    outer = max(cam.disk_outer_radius, inner * 1.0001)
    rh = m + math.sqrt(max(m * m - a * a, 0.0)) if abs(a) > 1e-12 else 2.0 * m
    r_obs = max(cam.observer_position[1], rh * 1.02)
    pixel = cam.field_of_view_rad / max(cam.screen_width, 1)
    detail = min(max((2.0 * rh / r_obs) / max(pixel * 24.0, 1e-9), 0.0), 1.0)
    return m, a, inner, outer, detail


def oracle_pixels(cam, sh, status, r_hit, phi, g):
    L = O.lib()
    prof_in = np.frombuffer(bytes(sh.disk), np.float32).copy()
    over = np.array([sh.disk_temperature_scale_k, sh.disk_temperature_floor_k, sh.disk_color_saturation,
                     sh.disk_doppler_beaming_exponent])
    prof = np.zeros(32, np.float32)
    L.orc_resolve_profile(O._p(prof_in), O._p(over), O._p(prof))
    m, a, inner, outer, detail = _camera_constants(cam)
    out = np.zeros((status.size, 3), np.float32)
    px = np.zeros(3, np.float32)
    for i in range(status.size):
        L.orc_shade_pixel(O._p(prof), sh.hydro_model, sh.accretion_rate_scale, sh.tonemapping_mode,
                          sh.camera_exposure, m, a, inner, outer, sh.time, detail, int(status[i]),
                          float(r_hit[i]), float(phi[i]), float(g[i]), O._p(px))
        out[i] = px
    return out


def oracle_cont_pixels(cam, sh, cont):
    """Pixels of the oracle's continuation trace: every recorded crossing
    shaded at the throughput left (orc_shade_cont)."""
    L = O.lib()
    prof_in = np.frombuffer(bytes(sh.disk), np.float32).copy()
    over = np.array([sh.disk_temperature_scale_k, sh.disk_temperature_floor_k, sh.disk_color_saturation,
                     sh.disk_doppler_beaming_exponent])
    prof = np.zeros(32, np.float32)
    L.orc_resolve_profile(O._p(prof_in), O._p(over), O._p(prof))
    m, a, inner, outer, detail = _camera_constants(cam)
    out = np.zeros((cont.size, 3), np.float32)
    px = np.zeros(3, np.float32)
    for i in range(cont.size):
        cr, cp, cg = (np.ascontiguousarray(cont[f][i]) for f in ("cross_r", "cross_phi", "cross_g"))
        L.orc_shade_cont(O._p(prof), sh.hydro_model, sh.accretion_rate_scale, sh.tonemapping_mode,
                         sh.camera_exposure, m, a, inner, outer, sh.time, detail, int(cont["n_cross"][i]),
                         O._p(cr), O._p(cp), O._p(cg), O._p(px))
        out[i] = px
    return out


def _rgb(pix):
    return np.stack([pix["r"], pix["g"], pix["b"]], 1)


SHADINGS = {
    "defaults": {},
    "novikov_thorne_aces": dict(hydro_model=1, tonemapping_mode=1, accretion_rate_scale=2.0, time=3.5),
    "log_exposure": dict(tonemapping_mode=2, camera_exposure=1.5, time=10.0),
    "reinhard_hot": dict(tonemapping_mode=3, disk_temperature_scale_k=40000.0, disk_doppler_beaming_exponent=3.0),
}


@pytest.mark.parametrize("name", list(SHADINGS))
def test_kerr_schild_pixels_match_oracle(tracer, name):
    """FP64 tracer through the translucent disk against the oracle's
    continuation trace (same algorithm): sRGB within CONT_BAR on every ray
    away from the critical curve and the disk edges."""
    cam = relsim.make_camera(spin=0.94, r_obs=40.0, incl_deg=70.0, fov_deg=30.0, width=64, height=64)
    sh = relsim.shading(**SHADINGS[name])
    tracer.set_shading(sh)
    try:
        out = tracer.dispatch(cam, fields=["status", "r_hit", "phi", "g"], pixels=True)
    finally:
        tracer.set_shading(None)
    rgb = _rgb(out["pixels"])
    ref, cont = O.trace_cont(relsim.camera_dict(cam))
    want = oracle_cont_pixels(cam, sh, cont)
    keep = ~(O.boundary_band(ref, _camera_constants(cam)[2], cam.disk_outer_radius) |
             (np.abs(ref["db_shadow"]) < 1e-3))
    disk = out["status"] == relsim.RAY_DISK
    assert disk.sum() > 500 and (cont["n_cross"] > 1).sum() > 100  # later crossings are seen
    err = np.abs(rgb - want).max(1)[keep]
    print(f"{name}: max sRGB difference {err.max():.2e} over {keep.sum()} rays")
    assert err.max() < CONT_BAR, err.max()
    np.testing.assert_array_equal(rgb[~disk], 0.0)
    np.testing.assert_array_equal(out["pixels"]["a"], 1.0)
    assert rgb[disk].max() > 0.05  # the disk is lit


def test_shading_leaves_the_record_unchanged(tracer):
    """The translucent-disk continuation follows rays on after their first hit;
    the record (and the pixel's iterations and affine parameter) still
    describes the first hit, bit for bit as an unshaded dispatch gives it.  A
    disk pixel's flags add the way the ray ended and its redshift is the last
    crossing's."""
    fields = ["status", "flags", "steps_accepted", "steps_rejected", "r", "theta", "phi", "r_hit", "g", "lambda",
              "dH", "dE", "dLz", "dQ"]
    for prec in (relsim.PRECISION_FP64, relsim.PRECISION_MIXED):
        cam = relsim.make_camera(spin=0.94, r_obs=40.0, incl_deg=70.0, fov_deg=30.0, width=48, height=48,
                                 precision=prec)
        plain = tracer.dispatch(cam, fields=fields, pixels=True)
        tracer.set_shading(relsim.shading(tonemapping_mode=1))
        try:
            shaded = tracer.dispatch(cam, fields=fields, pixels=True)
        finally:
            tracer.set_shading(None)
        for f in fields:
            np.testing.assert_array_equal(shaded[f], plain[f])
        for f in ("affine_parameter", "iterations_used"):
            np.testing.assert_array_equal(shaded["pixels"][f], plain["pixels"][f])
        disk = plain["status"] == relsim.RAY_DISK
        flags = shaded["pixels"]["status_flags"]
        assert np.all(flags[disk] & relsim.PIXEL_ACCRETION_DISK_HIT)
        np.testing.assert_array_equal(flags[~disk], plain["pixels"]["status_flags"][~disk])
        assert (flags[disk] != relsim.PIXEL_ACCRETION_DISK_HIT).sum() > 100  # rays that went on


def test_oracle_trace_shaded_matches_mixed(tracer):
    """The mixed tracer through the translucent disk against the FP64 oracle's
    continuation trace: its crossings lie within the mixed tracer's stated
    error, so pixels agree within MIXED_CONT_BAR away from the critical curve
    and the disk edges."""
    cam = relsim.make_camera(spin=0.9, r_obs=50.0, incl_deg=75.0, fov_deg=30.0, width=48, height=48,
                             precision=relsim.PRECISION_MIXED)
    sh = relsim.shading(hydro_model=1, tonemapping_mode=1)
    tracer.set_shading(sh)
    try:
        out = tracer.dispatch(cam, fields=["status"], pixels=True)
    finally:
        tracer.set_shading(None)
    ocam = relsim.make_camera(spin=0.9, r_obs=50.0, incl_deg=75.0, fov_deg=30.0, width=48, height=48)
    ref, cont = O.trace_cont(relsim.camera_dict(ocam))
    want = oracle_cont_pixels(ocam, sh, cont)
    keep = ~(O.boundary_band(ref, _camera_constants(ocam)[2], ocam.disk_outer_radius, 1e-3) |
             (np.abs(ref["db_shadow"]) < 1e-2))
    err = np.abs(_rgb(out["pixels"]) - want).max(1)[keep]
    assert err.max() < MIXED_CONT_BAR, err.max()


def test_boyer_lindquist_pixels_match_oracle(tracer):
    """Boyer-Lindquist Kerr-Newman tracer through the translucent disk against
    the oracle's continuation trace (same algorithm), same bars."""
    cam = relsim.make_camera(spin=0.9, r_obs=50.0, incl_deg=75.0, fov_deg=30.0, width=48, height=48,
                             metric_form=relsim.METRIC_BOYER_LINDQUIST, charge=0.3)
    sh = relsim.shading(tonemapping_mode=1)
    tracer.set_shading(sh)
    try:
        out = tracer.dispatch(cam, fields=["status", "r_hit", "phi", "g"], pixels=True)
    finally:
        tracer.set_shading(None)
    ref, cont = O.bl_trace_cont(relsim.camera_dict(cam), 0.3)
    want = oracle_cont_pixels(cam, sh, cont)
    keep = ~(O.boundary_band(ref, _camera_constants(cam)[2], cam.disk_outer_radius) |
             (np.abs(ref["db_shadow"]) < 1e-3))
    err = np.abs(_rgb(out["pixels"]) - want).max(1)[keep]
    assert err.max() < CONT_BAR, err.max()
    assert (out["status"] == relsim.RAY_DISK).sum() > 300 and (cont["n_cross"] > 1).sum() > 50


def test_device_entry_point_and_tiles(tracer):
    """rt_dispatch_device with only pixels asked for (the record fields come from
    the handle's scratch) and a tile give the host call's pixels."""
    import torch
    cam = relsim.make_camera(spin=0.94, r_obs=40.0, incl_deg=70.0, fov_deg=30.0, width=40, height=40)
    tracer.set_shading(relsim.shading(tonemapping_mode=1))
    try:
        host = tracer.dispatch(cam, fields=[], pixels=True)["pixels"]
        n = 40 * 40
        pix = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
        rc = tracer.lib.rt_dispatch_device(tracer._h, ctypes.byref(cam), pix.data_ptr(), None, n, None)
        assert rc == relsim.RT_OK
        assert tracer.lib.rt_synchronize(tracer._h, 0.0) == relsim.RT_OK
        dev = pix.cpu().numpy().view(relsim.PIXEL_DTYPE)
        np.testing.assert_array_equal(dev, host)
        tile = relsim.make_camera(spin=0.94, r_obs=40.0, incl_deg=70.0, fov_deg=30.0, width=40, height=40)
        tile.tile_origin_x, tile.tile_origin_y, tile.tile_extent_x, tile.tile_extent_y = 5, 12, 17, 9
        t = tracer.dispatch(tile, fields=[], pixels=True, tile=True)["pixels"]
        np.testing.assert_array_equal(t, host.reshape(40, 40)[12:21, 5:22].ravel())
    finally:
        tracer.set_shading(None)
    off = tracer.dispatch(cam, fields=[], pixels=True)["pixels"]
    np.testing.assert_array_equal(_rgb(off), 0.0)


def test_unsupported_settings_rejected(tracer):
    with pytest.raises(relsim.RelsimError):
        tracer.set_shading(relsim.shading(sky_enabled=1))
    with pytest.raises(relsim.RelsimError):
        tracer.set_shading(relsim.shading(hydro_model=2))
    with pytest.raises(relsim.RelsimError):
        tracer.set_shading(relsim.shading(tonemapping_mode=4))
