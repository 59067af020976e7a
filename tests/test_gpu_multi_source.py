"""Multi-source Kerr-Schild tracer (rt_dispatch_multi, csrc/rt_multi.cu)
against the FP64 multi-source oracle (oracle/ms_oracle.c, pinned to the
reference's multi-source functions by tests/test_oracle_multi_source.py).

Same algorithm on both sides (DP45 + PI30 + projection on the superposed
Hamiltonian, rtol = atol = 1e-10).  Bars:
  - class identical for at least 99.9 % of rays, and the DIVERGED flag equal
    on rays of equal class;
  - escaped and disk rays of equal class: final (r, theta, phi), disk radius
    and g within 1e-9 relative for 99.5 % of them and within 1e-6 for 99.9 %
    (measured: all within 2e-10 on B200; scenes of several holes scatter rays
    chaotically, so a near-critical ray amplifies last-bit differences of the
    kernel's rearranged RHS arithmetic, and a superposition has no critical
    curve to exclude such rays by, as the single-hole parity test does);
  - captured rays: class and flag only.  A capture ends at the first step end
    inside 1.01 r_+ of a source, or where |p| passes 1000 (DIVERGED), both
    points where the backward-traced ray is most sensitive to last-bit
    differences, so their positions are not compared;
  - accepted step counts within one of each other for 99 % of escaped and
    disk rays (with up to 16 sources summed, a last-bit difference now and then
    moves an acceptance decision at err = 1 by one step, about one ray in ten;
    the outcome stays within the bars above);
  - the per-ray constraint drift dH (the largest |H| of the superposed
    Hamiltonian before a projection; the Kerr invariants E, L_z, Q do not exist
    for a superposition and are NaN on both sides) within 1e-12 of the
    oracle's for 99.9 % of escaped and disk rays (measured on B200: 9e-16 at
    most over three stream scenes, with dH itself up to 5e-4).
"""
import numpy as np
import pytest

import relsim
import scenes
from cameras import config_cam
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ["status", "flags", "steps_accepted", "steps_rejected", "r", "theta", "phi", "r_hit", "g", "lambda",
          "dH", "dE", "dLz", "dQ", "exit_x", "exit_y", "exit_z"]


def same(a, b) -> bool:
    return np.array_equal(a, b, equal_nan=(a.dtype.kind == "f"))


def _oracle_sources(srcs):
    return [{"position": list(s.position), "mass": s.mass, "spin_parameter": s.spin_parameter, "axis": list(s.axis),
             "disk_enabled": s.disk_enabled, "disk_inner_scale": s.disk_inner_scale,
             "disk_outer_units": s.disk_outer_units} for s in srcs]


def _compare(tracer, cam, srcs):
    out = tracer.dispatch_multi(cam, srcs, fields=FIELDS, pixels=True)
    ref = O.ms_trace(relsim.camera_dict(cam), _oracle_sources(srcs))
    st, rst = out["status"], ref["status"]
    assert (st == rst).mean() >= 0.999, (st != rst).sum()
    eq = st == rst
    div, rdiv = out["flags"] & relsim.RAYFLAG_DIVERGED, ref["flags"] & relsim.RAYFLAG_DIVERGED
    assert (div[eq] == rdiv[eq]).mean() >= 0.999
    traced = eq & ((rst == O.ESCAPED) | (rst == O.DISK))
    dacc = np.abs(out["steps_accepted"].astype(np.int64) - ref["steps_accepted"].astype(np.int64))
    if traced.any():
        assert (dacc[traced] <= 1).mean() >= 0.99, (dacc[traced] <= 1).mean()
    same = traced

    def share_within(rel, tol):
        return float(np.mean(rel < tol)) if rel.size else 1.0

    for f in ("r", "theta", "phi"):
        floor = 1.0 if f == "phi" else 1e-300
        rel = np.abs(out[f][same] - ref[f][same]) / np.maximum(np.abs(ref[f][same]), floor)
        assert share_within(rel, 1e-9) >= 0.995, (f, share_within(rel, 1e-9))
        assert share_within(rel, 1e-6) >= 0.999, (f, share_within(rel, 1e-6))
    disk = same & (rst == O.DISK)
    for f in ("r_hit", "g"):
        rel = np.abs(out[f][disk] - ref[f][disk]) / ref[f][disk]
        assert share_within(rel, 1e-9) >= 0.995, (f, share_within(rel, 1e-9))
        assert share_within(rel, 1e-6) >= 0.999, (f, share_within(rel, 1e-6))
    dh = np.abs(out["dH"][same] - ref["dH"][same])
    assert share_within(dh, 1e-12) >= 0.999, share_within(dh, 1e-12)
    for f in ("dE", "dLz", "dQ"):
        assert np.all(np.isnan(out[f])), f
    # sky-lookup directions of escaped rays (the superposed flow), same bars
    esc = same & (rst == O.ESCAPED)
    e = np.stack([out["exit_x"], out["exit_y"], out["exit_z"]], 1)
    de = np.max(np.abs(e[esc] - ref["exit_dir"][esc]), axis=1) if esc.any() else np.zeros(0)
    assert share_within(de, 1e-9) >= 0.995 and share_within(de, 1e-6) >= 0.999
    assert np.all(np.isnan(e[st != O.ESCAPED]))
    assert np.all(out["status"] != relsim.RAY_UNFINISHED)
    return out, ref


def test_single_hole_scene_matches_oracle(tracer):
    _compare(tracer, config_cam("c2", width=48, height=48), [])


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_stream_scenes_match_oracle(tracer, k):
    """Multi-source requests of the seeded stream (2..16 holes), at 40^2."""
    req = [r for r in scenes.request_stream() if r.multi_source][k]
    cam = req.bundle.camera(relsim.PRECISION_FP64)
    cam.screen_width = cam.screen_height = 40
    out, ref = _compare(tracer, cam, scenes.rt_sources(req.sources))
    assert len(req.sources) >= 1


def test_hand_placed_binary_with_both_disks(tracer):
    cam = relsim.make_camera(spin=0.6, r_obs=60.0, incl_deg=70.0, fov_deg=35.0, width=48, height=48)
    srcs = [relsim.make_source((12.0, 6.0, -3.0), 0.5, 0.8, (0.3, 0.2, 1.0), disk_outer_units=16.0)]
    out, ref = _compare(tracer, cam, srcs)
    # both holes' disks are seen
    assert (out["status"] == relsim.RAY_DISK).sum() > 100


def test_invalid_sources_are_rejected(tracer):
    cam = config_cam("c2", width=8, height=8)
    with pytest.raises(relsim.RelsimError):
        tracer.dispatch_multi(cam, [relsim.make_source((1.0, 2.0, 3.0))] * 16)
    with pytest.raises(relsim.RelsimError):
        tracer.dispatch_multi(cam, [relsim.make_source((1.0, 2.0, 3.0), mass=0.0)])


def test_sixteen_holes_repeat_and_windows(tracer):
    """The largest scene (16 holes: the camera's and 15 bodies) matches the
    oracle; a repeated dispatch is bit-identical; a row window and the device
    entry point give the same records as the rows of the whole image."""
    import torch

    req = [r for r in scenes.request_stream() if r.multi_source and len(r.sources) == 15][0]
    cam = req.bundle.camera(relsim.PRECISION_FP64)
    cam.screen_width = cam.screen_height = 40
    srcs = scenes.rt_sources(req.sources)
    out, ref = _compare(tracer, cam, srcs)
    again = tracer.dispatch_multi(cam, srcs, fields=FIELDS, pixels=True)
    for f in FIELDS:
        np.testing.assert_array_equal(again[f], out[f])
    np.testing.assert_array_equal(again["pixels"], out["pixels"])
    win = req.bundle.camera(relsim.PRECISION_FP64)
    win.screen_width = win.screen_height = 40
    win.dispatch_row_offset, win.dispatch_row_count = 7, 11
    part = tracer.dispatch_multi(win, srcs, fields=FIELDS, pixels=False)
    for f in FIELDS:
        np.testing.assert_array_equal(part[f], out[f][7 * 40:18 * 40])
    n = 40 * 40
    ro, dev = relsim.device_ray_out(n, ["status", "r_hit", "phi"])
    tracer.dispatch_multi_device(cam, srcs, ro, None, n)
    tracer.synchronize()
    np.testing.assert_array_equal(dev["status"].cpu().numpy().view(np.uint32), out["status"])
    np.testing.assert_array_equal(dev["r_hit"].cpu().numpy(), out["r_hit"])
    np.testing.assert_array_equal(dev["phi"].cpu().numpy(), out["phi"])


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_mixed_stream_scenes_against_oracle(tracer, k):
    """The stream's multi-source requests as served (a mixed-mode camera: the
    multi-source tracer runs its FP64 stages at the mode's rtol = atol = 1e-8)
    at 64^2, against the FP64 multi-source oracle at rtol 1e-10: class
    identical for at least 99 % of rays; disk radius and g within 1e-6 for at
    least 99 % of the disk rays of equal class and within 1e-3 for 99.9 % (a
    superposition scatters rays chaotically and has no critical curve to
    exclude near-critical rays by)."""
    req = [r for r in scenes.request_stream() if r.multi_source][k]
    srcs = scenes.rt_sources(req.sources)
    cam = req.bundle.camera(relsim.PRECISION_MIXED)
    cam.screen_width = cam.screen_height = 64
    tracer.set_launch_config()
    out = tracer.dispatch_multi(cam, srcs, fields=["status", "r_hit", "g"], pixels=False)
    ref_cam = req.bundle.camera(relsim.PRECISION_FP64)
    ref_cam.screen_width = ref_cam.screen_height = 64
    ref = O.ms_trace(relsim.camera_dict(ref_cam), _oracle_sources(srcs))
    same = out["status"] == ref["status"]
    disk = same & (ref["status"] == O.DISK)
    rel = np.abs(out["r_hit"][disk] - ref["r_hit"][disk]) / ref["r_hit"][disk]
    relg = np.abs(out["g"][disk] - ref["g"][disk]) / ref["g"][disk]
    share = lambda v, t: float(np.mean(v < t)) if v.size else 1.0
    print(f"scene {k} ({len(srcs) + 1} holes): class {same.mean():.5f}, {rel.size} disk rays, r_hit within 1e-6 "
          f"{share(rel, 1e-6):.4f}, max {rel.max() if rel.size else 0:.2e}; g within 1e-6 {share(relg, 1e-6):.4f}")
    assert same.mean() >= 0.99
    assert share(rel, 1e-6) >= 0.99 and share(relg, 1e-6) >= 0.99
    assert share(rel, 1e-3) >= 0.999 and share(relg, 1e-3) >= 0.999


def _ms_oracle_pixels(cam, sh, srcs, cont):
    """Pixels of the multi-source oracle's continuation trace: each crossing, in
    order, shaded with its source's disk (the camera's hole: rt_shading's
    resolved profile; a body: its own profile as it stands) by the thin
    procedural model at detail 1, at the throughput left (trace_multi_source,
    software_compute_engine.hpp:3150-3191), then tonemapped."""
    L = O.lib()
    prof_in = np.frombuffer(bytes(sh.disk), np.float32).copy()
    over = np.array([sh.disk_temperature_scale_k, sh.disk_temperature_floor_k, sh.disk_color_saturation,
                     sh.disk_doppler_beaming_exponent])
    primary = np.zeros(32, np.float32)
    L.orc_resolve_profile(O._p(prof_in), O._p(over), O._p(primary))
    profiles = [primary] + [np.frombuffer(bytes(s.disk), np.float32).copy() for s in srcs]
    t = O.ms_table(relsim.camera_dict(cam), _oracle_sources(srcs))[0]
    out = np.zeros((cont.size, 3), np.float32)
    px = np.zeros(3, np.float32)
    shv = np.zeros(4)
    for i in range(cont.size):
        acc = np.zeros(3)
        thr = 1.0
        for k in range(int(cont["n_cross"][i])):
            if not thr > 0.01:
                break
            s = int(cont["cross_src"][i][k])
            pt = np.array([t["mass"][s], t["spin"][s], t["disk_in"][s], t["disk_out"][s], cont["cross_r"][i][k],
                           cont["cross_phi"][i][k], cont["cross_g"][i][k], sh.time, 1.0])
            L.orc_disk_shade(O._p(profiles[s]), O._p(pt), 0, sh.accretion_rate_scale, O._p(shv))
            acc += thr * shv[:3]
            thr *= 1.0 - shv[3]
        L.orc_tonemap(O._p(acc), sh.tonemapping_mode, sh.camera_exposure, O._p(px))
        out[i] = px
    return out


@pytest.mark.parametrize("k", [1, 2])
def test_multi_source_shaded_pixels_match_oracle(tracer, k):
    """Shaded multi-source scenes (the bodies' disks drawn with their own
    profiles, one body given a hotter, brighter disk): every ray followed
    through the translucent disks of all sources, the crossings composed in
    order.  Against the oracle's continuation trace shaded the same way: sRGB
    within 1e-5 for at least 99 % of the rays (the rest are rays that the
    superposed fields scatter chaotically, whose crossings differ), and the
    shaded dispatch's records equal the unshaded dispatch's bit for bit.  The
    body index of each record (the source of its first disk hit or capture)
    equals the oracle's on every ray of equal class."""
    req = [r for r in scenes.request_stream() if r.multi_source][k]
    srcs = scenes.rt_sources(req.sources)
    srcs[0].disk.peak_temperature_k = 30000.0
    srcs[0].disk.brightness = 1.5
    cam = req.bundle.camera(relsim.PRECISION_FP64)
    cam.screen_width = cam.screen_height = 40
    fields = ["status", "flags", "steps_accepted", "r", "theta", "phi", "r_hit", "g", "lambda", "dH", "body"]
    plain = tracer.dispatch_multi(cam, srcs, fields=fields, pixels=True)
    sh = relsim.shading(tonemapping_mode=1, time=2.0)
    tracer.set_shading(sh)
    try:
        shaded = tracer.dispatch_multi(cam, srcs, fields=fields, pixels=True)
    finally:
        tracer.set_shading(None)
    for f in fields:
        assert same(shaded[f], plain[f]), f
    ref, cont = O.ms_trace_cont(relsim.camera_dict(cam), _oracle_sources(srcs))
    eq = shaded["status"] == ref["status"]
    assert (shaded["body"][eq] == ref["body"][eq]).all()
    assert (shaded["body"][eq & (ref["status"] == O.DISK)] != relsim.BODY_NONE).all()
    want = _ms_oracle_pixels(cam, sh, srcs, cont)
    got = np.stack([shaded["pixels"]["r"], shaded["pixels"]["g"], shaded["pixels"]["b"]], 1)
    d = np.max(np.abs(got - want), axis=1)
    print(f"scene {k}: {int((cont['n_cross'] > 1).sum())} rays with 2+ crossings, sources crossed "
          f"{sorted(set(cont['cross_src'][cont['n_cross'] > 0][:, 0].tolist()))}; sRGB within 1e-5 "
          f"{np.mean(d < 1e-5):.4f}, max {d.max():.2e}")
    assert np.mean(d < 1e-5) >= 0.99
    assert (cont["n_cross"] > 1).any() and got.max() > 0.0


def test_multi_source_with_the_torus_model_drops_the_primary_disk(tracer):
    """Hydro model 2 in a multi-source scene: the reference's multi-source path
    draws no torus and turns the camera hole's disk off
    (software_compute_engine.hpp:2752), the bodies' disks shaded as usual.
    Against the oracle's continuation trace of the scene with the camera's
    disk off, composed the same way: sRGB within 1e-5 for 99 % of the rays."""
    req = [r for r in scenes.request_stream() if r.multi_source][1]
    srcs = scenes.rt_sources(req.sources)
    cam = req.bundle.camera(relsim.PRECISION_FP64)
    cam.screen_width = cam.screen_height = 40
    sh = relsim.shading(hydro_model=2, tonemapping_mode=1, time=2.0)
    tracer.set_shading(sh)
    try:
        shaded = tracer.dispatch_multi(cam, srcs, fields=["status", "body"], pixels=True)
    finally:
        tracer.set_shading(None)
    off = type(cam).from_buffer_copy(cam)
    off.disk_outer_radius = 0.0
    ref, cont = O.ms_trace_cont(relsim.camera_dict(off), _oracle_sources(srcs))
    eq = shaded["status"] == ref["status"]
    assert eq.mean() >= 0.99
    crossed = cont["n_cross"] > 0
    assert crossed.any() and (cont["cross_src"][crossed][:, 0] != 0).all()
    assert (shaded["body"][eq & (ref["status"] == O.DISK)] != 0).all()
    want = _ms_oracle_pixels(off, relsim.shading(tonemapping_mode=1, time=2.0), srcs, cont)
    got = np.stack([shaded["pixels"]["r"], shaded["pixels"]["g"], shaded["pixels"]["b"]], 1)
    d = np.max(np.abs(got - want), axis=1)
    print(f"torus model, multi-source: {int(crossed.sum())} rays cross a body's disk; sRGB within 1e-5 "
          f"{np.mean(d < 1e-5):.4f}, max {d.max():.2e}")
    assert np.mean(d < 1e-5) >= 0.99
