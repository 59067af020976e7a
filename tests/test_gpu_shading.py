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
disk hits are exactly black with alpha 1 when the sky is off.

With the sky on, a ray that escapes with throughput left adds the procedural
sky at its exit direction; the oracle side samples the reference's own
SkyboxRenderer::sample_sky (compiled from the reference headers into
oracle/_ref) at the oracle's exit direction.  Bar SKY_BAR (1e-6) in sRGB
for 99.5 % of the compared rays and SKY_MAX for every one: a point-like
star's flux changes as theta dtheta / sigma^2 with the 1e-9 rad difference
of the two traces' exit directions, and CUDA's transcendental functions
differ from the host's (measured on B200: every ray within 9e-7).
"""
import ctypes
import math
import os

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
        tracer.set_shading(relsim.shading(sky_enabled=2))
    with pytest.raises(relsim.RelsimError):
        tracer.set_shading(relsim.shading(hydro_model=3))
    with pytest.raises(relsim.RelsimError):
        tracer.set_shading(relsim.shading(tonemapping_mode=4))



SKY_BAR = 1e-6
SKY_MAX = 1e-4


@pytest.fixture(scope="module")
def sky_sampler(tmp_path_factory):
    """The sky the oracle side adds: the reference's SkyboxRenderer::sample_sky
    from oracle/_ref where that library was built; else the library's own sky
    arithmetic compiled for the host (tests/sky/sky_host.cpp), which
    tests/test_sky_host.py pins to the reference on every layer."""
    import subprocess
    v, d = ctypes.c_void_p, ctypes.c_double
    if O.ref_available():
        fn = O.ref().ref_sample_sky
        which = "reference"
    else:
        here = os.path.dirname(os.path.abspath(__file__))
        out = tmp_path_factory.mktemp("sky") / "libsky_host.so"
        subprocess.run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-I",
                        os.path.join(os.path.dirname(here), "relativity-simulator_b200", "csrc"),
                        os.path.join(here, "sky", "sky_host.cpp"), "-o", str(out)], check=True)
        fn = ctypes.CDLL(str(out)).host_sample_sky
        which = "host build"
    fn.argtypes = [v, d, d, d, d, d, v]
    fn.restype = None
    print(f"sky sampled by the {which}")
    return fn


def oracle_sky_pixels(sample, cam, sh, cont, srcs=None):
    """Pixels of an oracle continuation trace with the sky: the crossings shaded
    in order at the throughput left (the camera's disk, or each source's for a
    multi-source scene), then, for a ray that escaped with more than 0.01 of
    its throughput, the sky at the oracle's exit direction times that
    throughput; tonemapped.  NaN for rays the oracle left unfinished."""
    L = O.lib()
    prof_in = np.frombuffer(bytes(sh.disk), np.float32).copy()
    over = np.array([sh.disk_temperature_scale_k, sh.disk_temperature_floor_k, sh.disk_color_saturation,
                     sh.disk_doppler_beaming_exponent])
    primary = np.zeros(32, np.float32)
    L.orc_resolve_profile(O._p(prof_in), O._p(over), O._p(primary))
    if srcs is None:
        m, a, inner, outer, detail = _camera_constants(cam)
        geo, profiles, hydro = [(m, a, inner, outer)], [primary], sh.hydro_model
    else:
        from test_gpu_multi_source import _oracle_sources
        t = O.ms_table(relsim.camera_dict(cam), _oracle_sources(srcs))[0]
        geo = [(t["mass"][i], t["spin"][i], t["disk_in"][i], t["disk_out"][i]) for i in range(len(srcs) + 1)]
        profiles = [primary] + [np.frombuffer(bytes(s.disk), np.float32).copy() for s in srcs]
        detail, hydro = 1.0, 0
    prof = (ctypes.c_uint8 * 1808).from_buffer_copy(bytes(sh.sky))
    out = np.full((cont.size, 3), np.nan, np.float32)
    px = np.zeros(3, np.float32)
    rgb = np.zeros(3, np.float32)
    shv = np.zeros(4)
    for i in range(cont.size):
        fate = int(cont["fate"][i])
        if fate == O.UNFINISHED:
            continue
        acc = np.zeros(3)
        thr = 1.0
        for k in range(int(cont["n_cross"][i])):
            if not thr > 0.01:
                break
            s_idx = int(cont["cross_src"][i][k]) if srcs is not None else 0
            m, a, inner, outer = geo[s_idx]
            pt = np.array([m, a, inner, outer, cont["cross_r"][i][k], cont["cross_phi"][i][k], cont["cross_g"][i][k],
                           sh.time, detail])
            L.orc_disk_shade(O._p(profiles[s_idx]), O._p(pt), hydro, sh.accretion_rate_scale, O._p(shv))
            acc += thr * shv[:3]
            thr *= 1.0 - shv[3]
        if thr > 0.01 and fate == O.ESCAPED:
            e = cont["exit_dir"][i]
            sample(ctypes.addressof(prof), float(e[0]), float(e[1]), float(e[2]), cam.field_of_view_rad, sh.time,
                   rgb.ctypes.data)
            acc += thr * rgb.astype(np.float64)
        L.orc_tonemap(O._p(acc), sh.tonemapping_mode, sh.camera_exposure, O._p(px))
        out[i] = px
    return out


def _sky_check(got, want, what, bar=SKY_BAR, top=SKY_MAX):
    ok = ~np.isnan(want).any(1)
    err = np.abs(got - want).max(1)[ok]
    print(f"{what}: {ok.sum()} rays compared, sRGB within {bar:g}: {np.mean(err < bar):.4f}, max {err.max():.2e}")
    assert ok.sum() > 0.8 * want.shape[0]
    assert np.mean(err < bar) >= 0.995 and err.max() < top


def _shaded(tracer, sh, call):
    tracer.set_shading(sh)
    try:
        return call()
    finally:
        tracer.set_shading(None)


def test_sky_behind_kerr_schild_rays_matches_oracle(tracer, sky_sampler):
    """The default procedural sky (every layer the reference turns on by
    default) behind a Kerr-Schild image whose field of view takes in the sky
    around the hole and the sky lensed through the translucent disk."""
    cam = relsim.make_camera(spin=0.94, r_obs=40.0, incl_deg=70.0, fov_deg=60.0, width=64, height=64)
    sh = relsim.shading(tonemapping_mode=1, time=1.5, sky_enabled=1)
    out = _shaded(tracer, sh, lambda: tracer.dispatch(cam, fields=["status"], pixels=True))
    ref, cont = O.trace_cont(relsim.camera_dict(cam))
    want = oracle_sky_pixels(sky_sampler, cam, sh, cont)
    want[O.boundary_band(ref, _camera_constants(cam)[2], cam.disk_outer_radius) |
         (np.abs(ref["db_shadow"]) < 1e-3)] = np.nan
    got = _rgb(out["pixels"])
    _sky_check(got, want, "Kerr-Schild")
    esc = cont["fate"] == O.ESCAPED
    assert esc.sum() > 1000 and got[esc].max() > 0.05
    assert (out["pixels"]["status_flags"][esc & (cont["n_cross"] == 0)] & relsim.PIXEL_CELESTIAL_HIT).all()


def test_sky_behind_mixed_rays_matches_oracle(tracer, sky_sampler):
    """The mixed tracer's exit directions carry its stated error (FP32 far
    from the hole): against the FP64 oracle, MIXED_CONT_BAR for 99.5 % of the
    rays, away from the critical curve and the disk edges."""
    kw = dict(spin=0.94, r_obs=40.0, incl_deg=70.0, fov_deg=60.0, width=64, height=64)
    cam = relsim.make_camera(precision=relsim.PRECISION_MIXED, **kw)
    sh = relsim.shading(tonemapping_mode=1, time=1.5, sky_enabled=1)
    out = _shaded(tracer, sh, lambda: tracer.dispatch(cam, fields=["status"], pixels=True))
    ocam = relsim.make_camera(**kw)
    ref, cont = O.trace_cont(relsim.camera_dict(ocam))
    want = oracle_sky_pixels(sky_sampler, ocam, sh, cont)
    want[O.boundary_band(ref, _camera_constants(ocam)[2], ocam.disk_outer_radius, 1e-3) |
         (np.abs(ref["db_shadow"]) < 1e-2)] = np.nan
    _sky_check(_rgb(out["pixels"]), want, "mixed", MIXED_CONT_BAR, 1e-2)


def test_sky_behind_boyer_lindquist_rays_matches_oracle(tracer, sky_sampler):
    """A Kerr-Newman Boyer-Lindquist image with a sky of other models: stars
    with diffraction spikes, denser galaxies and the coordinate grid."""
    cam = relsim.make_camera(spin=0.9, r_obs=50.0, incl_deg=75.0, fov_deg=40.0, width=48, height=48,
                             metric_form=relsim.METRIC_BOYER_LINDQUIST, charge=0.3)
    sky = relsim.sky_profile(star_profile_model=5, galaxy_density=1.5, grid_enabled=1, grid_show_equator=1)
    sh = relsim.shading(sky_enabled=1, sky=sky, time=0.5)
    out = _shaded(tracer, sh, lambda: tracer.dispatch(cam, fields=["status"], pixels=True))
    ref, cont = O.bl_trace_cont(relsim.camera_dict(cam), 0.3)
    want = oracle_sky_pixels(sky_sampler, cam, sh, cont)
    want[O.boundary_band(ref, _camera_constants(cam)[2], cam.disk_outer_radius) |
         (np.abs(ref["db_shadow"]) < 1e-3)] = np.nan
    _sky_check(_rgb(out["pixels"]), want, "Boyer-Lindquist")


def test_sky_behind_multi_source_rays_matches_oracle(tracer, sky_sampler):
    """The default sky behind a multi-source scene: each body's disk shaded
    with its own profile, the sky at the superposed flow's exit direction."""
    import scenes
    req = [r for r in scenes.request_stream() if r.multi_source][2]
    srcs = scenes.rt_sources(req.sources)
    cam = req.bundle.camera(relsim.PRECISION_FP64)
    cam.screen_width = cam.screen_height = 40
    sh = relsim.shading(sky_enabled=1, tonemapping_mode=3, time=4.0)
    out = _shaded(tracer, sh, lambda: tracer.dispatch_multi(cam, srcs, fields=["status"], pixels=True))
    from test_gpu_multi_source import _oracle_sources
    ref, cont = O.ms_trace_cont(relsim.camera_dict(cam), _oracle_sources(srcs))
    want = oracle_sky_pixels(sky_sampler, cam, sh, cont, srcs)
    want[out["status"] != ref["status"]] = np.nan
    _sky_check(_rgb(out["pixels"]), want, "multi-source")


def test_server_refuses_the_sky():
    with relsim.Server(0, relsim.server_config(1 << 26)) as srv:
        with pytest.raises(relsim.RelsimError):
            srv.set_shading(relsim.shading(sky_enabled=1))


def _resolved_profile(sh):
    prof_in = np.frombuffer(bytes(sh.disk), np.float32).copy()
    over = np.array([sh.disk_temperature_scale_k, sh.disk_temperature_floor_k, sh.disk_color_saturation,
                     sh.disk_doppler_beaming_exponent])
    out = np.zeros(32, np.float32)
    O.lib().orc_resolve_profile(O._p(prof_in), O._p(over), O._p(out))
    return out


@pytest.mark.parametrize("sky", [0, 1])
def test_torus_pixels_match_oracle(tracer, sky_sampler, sky):
    """Hydro model 2, the Fishbone-Moncrief torus: the FP64 Kerr-Schild tracer
    gathers each step's chord through the torus (no thin disk, no early
    capture), against the oracle's trace that does the same
    (orc_trace_volume, its torus pinned to the reference's HydroDiskContext by
    tests/test_oracle_torus.py), composed with the sky behind it when on.  A
    mixed-precision camera traces the same (hydro model 2 uses the FP64
    tracer at the camera's tolerances).  Bar: sRGB within 1e-6 for 99 % of
    the rays away from the shadow's edge and 1e-4 for all (a chord whose
    length rounds to another sample count differs a little more)."""
    kw = dict(spin=0.6, r_obs=60.0, incl_deg=75.0, fov_deg=50.0, width=40, height=40)
    cam = relsim.make_camera(**kw)
    sh = relsim.shading(hydro_model=2, tonemapping_mode=1, sky_enabled=sky, torus_inner_radius=6.0,
                        torus_center_radius=10.0, time=0.5)
    out = _shaded(tracer, sh, lambda: tracer.dispatch(cam, fields=["status", "r"], pixels=True))
    ocam = relsim.camera_dict(cam)
    ocam["disk_outer_radius"] = 0.0
    ocam["early_capture"] = 0
    m, a = _camera_constants(cam)[:2]
    fm = O.fm_context(m, a, (sh.torus_inner_radius, sh.torus_center_radius, sh.adiabatic_index,
                             sh.optical_depth_scale, sh.sampling_density), _resolved_profile(sh))
    ref, cont, vol = O.trace_volume(ocam, fm)
    np.testing.assert_array_equal(out["status"], ref["status"])
    prof = (ctypes.c_uint8 * 1808).from_buffer_copy(bytes(sh.sky))
    want = np.full((cont.size, 3), np.nan, np.float32)
    px = np.zeros(3, np.float32)
    rgb = np.zeros(3, np.float32)
    for i in range(cont.size):
        seen = vol[i, 5] != 0.0
        acc = vol[i, :3].copy() if seen else np.zeros(3)
        thr = vol[i, 3] if seen else 1.0
        if sky and thr > 0.01 and cont["fate"][i] == O.ESCAPED:
            e = cont["exit_dir"][i]
            sky_sampler(ctypes.addressof(prof), float(e[0]), float(e[1]), float(e[2]), cam.field_of_view_rad, sh.time,
                        rgb.ctypes.data)
            acc = acc + thr * rgb.astype(np.float64)
        O.lib().orc_tonemap(O._p(acc), sh.tonemapping_mode, sh.camera_exposure, O._p(px))
        want[i] = px
    want[np.abs(ref["db_shadow"]) < 1e-3] = np.nan
    got = _rgb(out["pixels"])
    ok = ~np.isnan(want).any(1)
    err = np.abs(got - want).max(1)[ok]
    seen = vol[:, 5] != 0.0
    print(f"torus (sky {sky}): {seen.sum()} rays through the torus, sRGB within 1e-6 {np.mean(err < 1e-6):.4f}, "
          f"max {err.max():.2e}")
    assert seen.sum() > 200 and np.mean(err < 1e-6) >= 0.99 and err.max() < 1e-4
    flags = out["pixels"]["status_flags"]
    assert ((flags & relsim.PIXEL_ACCRETION_DISK_HIT) != 0).tolist() == seen.tolist()
    z = out["pixels"]["redshift"][seen]
    assert np.allclose(z, vol[seen, 4].astype(np.float32), rtol=1e-5)
    # a mixed-precision camera: the FP64 tracer at its tolerance (1e-8)
    mixed = relsim.make_camera(precision=relsim.PRECISION_MIXED, **kw)
    fp64 = relsim.make_camera(rtol=mixed.rtol, **kw)
    a = _shaded(tracer, sh, lambda: tracer.dispatch(mixed, fields=["status", "r"], pixels=True))
    b = _shaded(tracer, sh, lambda: tracer.dispatch(fp64, fields=["status", "r"], pixels=True))
    np.testing.assert_array_equal(a["pixels"], b["pixels"])
    np.testing.assert_array_equal(a["r"], b["r"])


def test_torus_boyer_lindquist_pixels_match_oracle(tracer):
    """The torus behind a Kerr-Newman Boyer-Lindquist camera: each step's chord
    between its Boyer-Lindquist points, L / E as u^phi r^2 sin^2 theta at the
    step's end (the reference's metric-type path), against the oracle's BL
    trace that gathers the same; same bars as the Kerr-Schild test."""
    kw = dict(spin=0.6, r_obs=60.0, incl_deg=75.0, fov_deg=50.0, width=40, height=40,
              metric_form=relsim.METRIC_BOYER_LINDQUIST, charge=0.3)
    cam = relsim.make_camera(**kw)
    sh = relsim.shading(hydro_model=2, tonemapping_mode=1, torus_inner_radius=6.0, torus_center_radius=10.0)
    out = _shaded(tracer, sh, lambda: tracer.dispatch(cam, fields=["status"], pixels=True))
    ocam = relsim.camera_dict(cam)
    ocam["disk_outer_radius"] = 0.0
    ocam["early_capture"] = 0
    m, a = _camera_constants(cam)[:2]
    fm = O.fm_context(m, a, (sh.torus_inner_radius, sh.torus_center_radius, sh.adiabatic_index,
                             sh.optical_depth_scale, sh.sampling_density), _resolved_profile(sh))
    ref, cont, vol = O.bl_trace_volume(ocam, 0.3, fm)
    np.testing.assert_array_equal(out["status"], ref["status"])
    want = np.zeros((cont.size, 3), np.float32)
    px = np.zeros(3, np.float32)
    for i in range(cont.size):
        acc = vol[i, :3].copy() if vol[i, 5] != 0.0 else np.zeros(3)
        O.lib().orc_tonemap(O._p(acc), sh.tonemapping_mode, sh.camera_exposure, O._p(px))
        want[i] = px
    keep = np.abs(ref["db_shadow"]) >= 1e-3
    err = np.abs(_rgb(out["pixels"]) - want).max(1)[keep]
    seen = vol[:, 5] != 0.0
    print(f"torus, Boyer-Lindquist: {seen.sum()} rays through the torus, sRGB within 1e-6 "
          f"{np.mean(err < 1e-6):.4f}, max {err.max():.2e}")
    assert seen.sum() > 200 and np.mean(err < 1e-6) >= 0.99 and err.max() < 1e-4


def test_torus_model_refused_by_the_server():
    with relsim.Server(0, relsim.server_config(1 << 26)) as srv:
        with pytest.raises(relsim.RelsimError):
            srv.set_shading(relsim.shading(hydro_model=2))


def test_headline_image_with_the_sky_matches_oracle_sample(tracer, sky_sampler):
    """The headline image (Kerr a = 0.94, 2048^2, mixed precision) shaded as the
    bench's end-to-end number is (translucent disk, the default sky, ACES),
    through rt_dispatch into host pixels: 3,000 random pixels against the FP64
    oracle's continuation traces composed with the reference's sky, away from
    the critical curve and the disk edges.  Bars of the mixed tracer: sRGB
    within MIXED_CONT_BAR for 99.5 % of the sample, 1e-2 for all."""
    cam = relsim.make_camera(width=2048, height=2048, precision=relsim.PRECISION_MIXED)
    sh = relsim.shading(tonemapping_mode=1, sky_enabled=1)
    out = _shaded(tracer, sh, lambda: tracer.dispatch(cam, fields=["status"], pixels=True))
    ocam = relsim.make_camera(width=2048, height=2048)
    rng = np.random.default_rng(7)
    pix = np.sort(rng.choice(2048 * 2048, 3000, replace=False)).astype(np.uint64)
    ref, cont = O.trace_cont(relsim.camera_dict(ocam), pixels=pix)
    want = oracle_sky_pixels(sky_sampler, ocam, sh, cont)
    want[O.boundary_band(ref, _camera_constants(ocam)[2], ocam.disk_outer_radius, 1e-3) |
         (np.abs(ref["db_shadow"]) < 1e-2)] = np.nan
    got = _rgb(out["pixels"][pix.astype(np.int64)])
    _sky_check(got, want, "headline 2048^2 sample", MIXED_CONT_BAR, 1e-2)
    sky_seen = (cont["fate"] == O.ESCAPED)
    assert sky_seen.mean() > 0.5
