"""Boyer-Lindquist Kerr-Newman tracer (metric_form RT_METRIC_BOYER_LINDQUIST,
csrc/rt_bl.cu) against the FP64 oracle (oracle/bl_oracle.c, pinned to the
reference's KerrNewmanMetric, Christoffel symbols, ZAMO ray and RK45
integrator by tests/test_oracle_boyer_lindquist.py).

Same algorithm on both sides (DP45 + PI30 + u^t projection, rtol = atol =
1e-10).  Bars:
  - class identical outside the 1e-6 M boundary band (the Kerr-Newman critical
    curve and the disk edges);
  - escaped and disk rays of equal class: final (r, theta, phi), r_hit and g
    within 1e-9 relative for 99.5 % of them and 1e-6 for all;
  - accepted step counts equal for 99 % of rays (the kernel forms 1/rho^2,
    1/Delta and 1/(Delta sin^2) from one reciprocal, the oracle divides three
    times, so an acceptance decision at err = 1 can move by one step);
  - invariant drift dE within 1e-9 (1e-8 for the near-extremal hole, 1e-6 for
    rays captured at 1.01 r_+);
  - the per-ray drift itself (dH, dE, dLz, dQ) against the oracle's, ray by
    ray on escaped and disk rays away from the critical curve (|d_b| > 1e-3 M),
    absolutely: dH 1e-12, dE 1e-11, dLz 1e-10, dQ 1e-9 (largest differences
    measured on B200 over five cameras at 48^2: 9e-14, 1.1e-12, 1.1e-11,
    1.8e-10).
Also: row windows and tiles equal to the full image, determinism, the server,
and the argument checks (no horizon, bundles).
"""
import ctypes

import numpy as np
import pytest

import relsim
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ["status", "flags", "steps_accepted", "steps_rejected", "r", "theta", "phi", "r_hit", "g", "lambda", "dH",
          "dE", "dLz", "dQ"]

# absolute bars on the per-ray drift against the oracle's (same algorithm)
DRIFT_BARS = {"dH": 1e-12, "dE": 1e-11, "dLz": 1e-10, "dQ": 1e-9}

# spin, charge, camera keywords
CASES = {
    "kn": (0.9, 0.3, dict(r_obs=50.0, incl_deg=75.0, fov_deg=30.0)),
    "kerr_headline": (0.94, 0.0, dict(r_obs=100.0, incl_deg=17.0, fov_deg=12.0)),
    "schw": (0.0, 0.0, dict(r_obs=50.0, incl_deg=60.0, fov_deg=30.0, disk_inner=6.0)),
    "kn_hi_q": (0.5, 0.7, dict(r_obs=50.0, incl_deg=85.0, fov_deg=30.0)),
    "kn_retro": (-0.8, 0.4, dict(r_obs=30.0, incl_deg=45.0, fov_deg=40.0)),
}


def bl_cam(tag, side=64, **over):
    spin, charge, kw = CASES[tag]
    kw = dict(kw)
    kw.update(over)
    return relsim.make_camera(spin=spin, width=side, height=side, metric_form=relsim.METRIC_BOYER_LINDQUIST,
                              charge=charge, **kw)


def _r_in(cam):
    return cam.disk_inner_radius if cam.disk_inner_radius > 0 else relsim.lib().rt_kerr_isco_radius(1.0, cam.metric_spin)


def _compare(tracer, cam, de_far=1e-9):
    out = tracer.dispatch(cam, fields=FIELDS, pixels=True)
    ref = O.bl_trace(relsim.camera_dict(cam), cam.metric_charge)
    band = O.boundary_band(ref, _r_in(cam), cam.disk_outer_radius)
    st, rst = out["status"], ref["status"]
    np.testing.assert_array_equal(st[~band], rst[~band])
    assert np.all(st != relsim.RAY_UNFINISHED)
    same = (st == rst) & ~band & ((rst == O.ESCAPED) | (rst == O.DISK))

    def check(rel):
        if rel.size == 0:
            return
        assert np.mean(rel < 1e-9) >= 0.995, np.mean(rel < 1e-9)
        assert np.all(rel < 1e-6), rel.max()

    for f in ("r", "theta", "phi"):
        floor = 1.0 if f == "phi" else 1e-300
        check(np.abs(out[f][same] - ref[f][same]) / np.maximum(np.abs(ref[f][same]), floor))
    disk = same & (rst == O.DISK)
    for f in ("r_hit", "g"):
        check(np.abs(out[f][disk] - ref[f][disk]) / ref[f][disk])
    eq = (st == rst) & ~band
    assert np.mean(out["steps_accepted"][eq] == ref["steps_accepted"][eq]) >= 0.99
    ok = eq & (out["flags"] == 0)
    drift = same & (out["flags"] == 0) & (ref["flags"] == 0) & (np.abs(ref["db_shadow"]) > 1e-3)
    for f, bar in DRIFT_BARS.items():
        d = np.abs(out[f][drift] - ref[f][drift])
        assert d.max(initial=0.0) < bar, (f, float(d.max(initial=0.0)))
    assert np.max(np.abs(out["dE"][ok & (st != relsim.RAY_CAPTURED)]), initial=0.0) < de_far
    # captured at 1.01 r_+: u^t ~ 1/Delta there, and E = -u_t cancels between large terms
    assert np.max(np.abs(out["dE"][ok]), initial=0.0) < 1e-6
    # pixel output: status flags, redshift and affine parameter of the record
    pix = out["pixels"]
    flag = np.select([st == 1, st == 2, st == 3], [1, 2, 4], 0)
    np.testing.assert_array_equal(pix["status_flags"], flag)
    np.testing.assert_array_equal(pix["redshift"], out["g"].astype(np.float32))
    np.testing.assert_array_equal(pix["affine_parameter"], (-out["lambda"]).astype(np.float32))
    return out, ref


@pytest.mark.parametrize("tag", list(CASES))
def test_matches_oracle(tracer, tag):
    _compare(tracer, bl_cam(tag))


def test_early_capture_off_matches_oracle(tracer):
    _compare(tracer, bl_cam("kn", early_capture=False))


def test_no_disk_matches_oracle(tracer):
    out, ref = _compare(tracer, bl_cam("kn_hi_q", disk_outer=0.0))
    assert np.sum(out["status"] == relsim.RAY_CAPTURED) > 100


def test_schwarzschild_equals_zero_charge_kerr_newman(tracer):
    """a = Q = 0 through the Boyer-Lindquist form (metric type 1) reproduces
    itself bit for bit, and its image is left-right symmetric about the
    observer's meridian."""
    cam = bl_cam("schw", side=48, incl_deg=90.0)
    a = tracer.dispatch(cam, fields=["status", "r_hit"], pixels=False)
    st = a["status"].reshape(48, 48)
    np.testing.assert_array_equal(st, st[:, ::-1])
    np.testing.assert_array_equal(st, st[::-1, :])


def test_windows_and_tiles_equal_full_image(tracer):
    cam = bl_cam("kn", side=64)
    full = tracer.dispatch(cam, fields=["status", "r", "r_hit", "steps_accepted"], pixels=True)
    win = bl_cam("kn", side=64, row_offset=20, row_count=17)
    w = tracer.dispatch(win, fields=["status", "r", "r_hit", "steps_accepted"], pixels=True)
    sl = slice(20 * 64, 37 * 64)
    for k in ("status", "r", "steps_accepted"):
        np.testing.assert_array_equal(w[k], full[k][sl])
    np.testing.assert_array_equal(w["pixels"], full["pixels"][sl])
    tile = bl_cam("kn", side=64)
    tile.tile_origin_x, tile.tile_origin_y, tile.tile_extent_x, tile.tile_extent_y = 10, 30, 21, 9
    t = tracer.dispatch(tile, fields=["status", "r"], pixels=False, tile=True)
    ref = full["status"].reshape(64, 64)[30:39, 10:31].ravel()
    np.testing.assert_array_equal(t["status"], ref)
    np.testing.assert_array_equal(t["r"], full["r"].reshape(64, 64)[30:39, 10:31].ravel())


def test_deterministic(tracer):
    cam = bl_cam("kn_retro", side=48)
    a = tracer.dispatch(cam, fields=FIELDS, pixels=True)
    b = tracer.dispatch(cam, fields=FIELDS, pixels=True)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_device_entry_point_matches_host(tracer):
    import torch
    cam = bl_cam("kn", side=40)
    host = tracer.dispatch(cam, fields=["status", "r_hit"], pixels=False)
    n = 40 * 40
    st = torch.empty(n, dtype=torch.int32, device="cuda")
    rh = torch.empty(n, dtype=torch.float64, device="cuda")
    ro = relsim.RayOut()
    ro.status, ro.r_hit = st.data_ptr(), rh.data_ptr()
    rc = tracer.lib.rt_dispatch_device(tracer._h, ctypes.byref(cam), None, ctypes.byref(ro), n, None)
    assert rc == relsim.RT_OK
    assert tracer.lib.rt_synchronize(tracer._h, 0.0) == relsim.RT_OK
    np.testing.assert_array_equal(st.cpu().numpy().view(np.uint32), host["status"])
    np.testing.assert_array_equal(rh.cpu().numpy(), host["r_hit"])


def test_argument_checks(tracer):
    # no horizon: a^2 + Q^2 >= M^2
    cam = bl_cam("kn", side=8)
    cam.metric_charge = 0.5  # 0.9^2 + 0.5^2 > 1
    with pytest.raises(relsim.RelsimError) as e:
        tracer.dispatch(cam, fields=["status"], pixels=False)
    assert e.value.status == 1
    cam.metric_charge = float("nan")
    with pytest.raises(relsim.RelsimError):
        tracer.dispatch(cam, fields=["status"], pixels=False)
    bad = bl_cam("kn", side=8)
    bad.metric_form = 7
    with pytest.raises(relsim.RelsimError):
        tracer.dispatch(bad, fields=["status"], pixels=False)
    # Boyer-Lindquist cameras are not bundle cameras
    import torch
    cams = (relsim.Camera * 1)(bl_cam("kn", side=8))
    st = torch.empty(64, dtype=torch.int32, device="cuda")
    ro = relsim.RayOut()
    ro.status = st.data_ptr()
    rc = tracer.lib.rt_trace_bundles_device(tracer._h, cams, 1, None, None, ctypes.byref(ro), 64, None)
    assert rc == 1


def test_server_request_matches_dispatch(tracer):
    """Boyer-Lindquist requests run in their own epochs beside Kerr-Schild ones
    and give the same records as a direct dispatch."""
    cam = bl_cam("kn", side=48)
    keys = ("status", "r", "r_hit", "g")
    ref = tracer.dispatch(cam, fields=list(keys), pixels=True)
    cfg = relsim.server_config(1 << 28, record=keys + ("pixels",))
    with relsim.Server(0, cfg) as srv:
        ks = relsim.make_camera(spin=0.9, width=32, height=32)
        a, oa = srv.submit(cam, keys, pixels=True)
        b, _ = srv.submit(ks, keys, pixels=True)
        c, oc = srv.submit(cam, keys, pixels=True)
        done = srv.wait([a, b, c])
    for rid, o in ((a, oa), (c, oc)):
        assert done[rid].status == relsim.RT_OK
        for k in keys:
            np.testing.assert_array_equal(o[k], ref[k])
        np.testing.assert_array_equal(o["pixels"], ref["pixels"])
    assert done[b].status == relsim.RT_OK


def test_server_rejects_invalid_boyer_lindquist(tracer):
    cam = bl_cam("kn", side=8)
    cam.metric_charge = 0.9  # no horizon
    with relsim.Server(0, relsim.server_config(1 << 26)) as srv:
        with pytest.raises(relsim.RelsimError) as e:
            srv.submit(cam)
        assert e.value.status == 1
        with pytest.raises(relsim.RelsimError):
            srv.submit(bl_cam("kn", side=8), sources=[relsim.make_source((10.0, 0.0, 0.0), 0.5, 0.3, (0, 0, 1))])


EDGE_CASES = {
    # observer 0.6 deg off the axis: rays pass the pole and are reflected
    "near_axis": (0.9, 0.3, dict(r_obs=30.0, incl_deg=0.6, fov_deg=40.0)),
    # close observer inside the disk's outer radius
    "close": (0.7, 0.5, dict(r_obs=5.0, incl_deg=60.0, fov_deg=90.0)),
    # near-extremal: a^2 + Q^2 = 0.9925 M^2, r_+ = 1.087 M
    "near_extremal": (0.95, 0.3, dict(r_obs=40.0, incl_deg=80.0, fov_deg=25.0)),
}


@pytest.mark.parametrize("tag", list(EDGE_CASES))
def test_edge_cases_match_oracle(tracer, tag):
    spin, charge, kw = EDGE_CASES[tag]
    cam = relsim.make_camera(spin=spin, width=48, height=48, metric_form=relsim.METRIC_BOYER_LINDQUIST, charge=charge,
                             **kw)
    # near-extremal: the steep near-horizon field drifts E by up to ~1.3e-9 on escaped and disk rays
    _compare(tracer, cam, de_far=1e-8 if tag == "near_extremal" else 1e-9)


def test_charge_sign_does_not_matter(tracer):
    """The Kerr-Newman metric depends on Q^2 only."""
    a = tracer.dispatch(bl_cam("kn_hi_q", side=32), fields=FIELDS, pixels=True)
    neg = bl_cam("kn_hi_q", side=32)
    neg.metric_charge = -neg.metric_charge
    b = tracer.dispatch(neg, fields=FIELDS, pixels=True)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
