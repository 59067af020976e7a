"""Continuous-batching request server (rt_server_*) on the GPU.

  - records equal a direct trace of the same camera (rt_dispatch);
  - a request's records are the same alone and inside a mix of concurrent
    requests of other sizes and both precisions (rays never share a warp with
    another request's rays: row chunks of widths that are multiples of 32 start
    on warp boundaries, so even the mixed mode's warp-uniform precision choice
    repeats; bit-identical);
  - admission holds the device-memory budget (peak records in use <= budget,
    requests wait until room frees up, then all complete);
  - a request larger than the budget is refused (BUDGET), a full queue answers
    AGAIN;
  - a multi-source request gives the same records through the server as
    through rt_dispatch_multi;
  - a short replay of the seeded request stream serves every request (single-
    and multi-source), with sampled rays within the mixed mode's stated error.
"""
import numpy as np
import pytest

import relsim
import scenes
from cameras import config_cam

pytestmark = pytest.mark.gpu

FIELDS = ("status", "r", "theta", "phi", "r_hit", "g")


def same(a, b) -> bool:
    return np.array_equal(a, b, equal_nan=(a.dtype.kind == "f"))


def _server(budget=1 << 28, **kw):
    return relsim.Server(0, relsim.server_config(budget, record=FIELDS + ("pixels",), **kw))


def test_server_matches_direct_trace(tracer):
    cams = [config_cam("c2", width=256, height=192, precision=relsim.PRECISION_MIXED),
            config_cam("c3", width=160, height=96),
            config_cam("c1", width=100, height=60),  # width not a multiple of 32
            config_cam("c2", width=64, height=64, row_offset=10, row_count=20)]
    tracer.set_launch_config()
    with _server() as srv:
        subs = [srv.submit(c, FIELDS, pixels=True) for c in cams]
        got = srv.wait([rid for rid, _ in subs])
        assert all(d.status == 0 for d in got.values())
    for cam, (rid, out) in zip(cams, subs):
        ref = tracer.dispatch(cam, fields=list(FIELDS), pixels=True)
        for k in FIELDS:
            assert same(out[k], ref[k]), k
        assert np.array_equal(out["pixels"], ref["pixels"])


@pytest.mark.parametrize("precision", [relsim.PRECISION_FP64, relsim.PRECISION_MIXED])
def test_request_same_alone_and_in_the_mix(precision):
    target = config_cam("c2", width=512, height=384, precision=precision)
    with _server(chunk_rays=1 << 15) as srv:
        rid, alone = srv.submit(target, FIELDS)
        srv.wait([rid])
    others = [d.camera(relsim.PRECISION_MIXED if i % 2 else relsim.PRECISION_FP64)
              for i, d in enumerate(scenes.bundle_table(24, 11)) if d.side <= 512]
    with _server(chunk_rays=1 << 15) as srv:
        ids = [srv.submit(c, FIELDS)[0] for c in others[:8]]
        rid, mixed_in = srv.submit(target, FIELDS)
        ids += [srv.submit(c, FIELDS)[0] for c in others[8:]]
        got = srv.wait(ids + [rid])
        st = srv.stats()
    assert all(d.status == 0 for d in got.values())
    assert st.peak_active > 1 and st.epochs > 1
    for k in FIELDS:
        assert same(mixed_in[k], alone[k]), k


def test_admission_holds_the_budget():
    cam = config_cam("c2", width=256, height=256)
    per_request = 256 * 256 * (4 + 5 * 8 + 32)
    budget = int(2.5 * per_request)
    with _server(budget) as srv:
        subs = [srv.submit(cam, FIELDS, pixels=True) for _ in range(8)]
        got = srv.wait([rid for rid, _ in subs])
        st = srv.stats()
    assert all(d.status == 0 for d in got.values())
    assert st.peak_bytes_in_use <= st.budget_bytes <= budget
    assert st.peak_active <= 2
    for _, out in subs[1:]:
        assert same(out["r_hit"], subs[0][1]["r_hit"])
    # later requests queued behind the budget: their latency includes the wait
    lat = sorted(d.latency_ms for d in got.values())
    assert lat[-1] > lat[0]


def test_oversized_request_and_full_queue():
    with _server(1 << 20) as srv:  # about 13 k rays of records
        with pytest.raises(relsim.RelsimError) as e:
            srv.submit(config_cam("c2", width=256, height=256), FIELDS)
        assert e.value.status == 7  # BUDGET
    with _server(1 << 30, max_requests=2) as srv:
        big = config_cam("c2", width=1024, height=1024)
        a, _ = srv.submit(big, FIELDS)
        b, _ = srv.submit(big, FIELDS)
        with pytest.raises(relsim.RelsimError) as e:
            srv.submit(big, FIELDS)
        assert e.value.status == 8  # AGAIN
        srv.wait([a, b])


def test_stream_replay_serves_every_request():
    import serve_stream

    reqs = scenes.request_stream(80)
    keep = {r.index for r in reqs[:40] if not r.multi_source}
    keep = set(sorted(keep)[:4])
    cfg = relsim.server_config(8 << 30, record=serve_stream.FIELDS)
    with relsim.Server(0, cfg) as srv:
        res = serve_stream.replay(srv, reqs, relsim.PRECISION_MIXED, speed=4.0, keep=keep)
    assert res["failed"] == 0
    assert res["served"] == len(reqs) and res["multi_source"] > 0
    assert res["latency_ms_p99"] >= res["latency_ms_p50"] > 0.0
    from oracle import oracle as O
    rng = np.random.default_rng(4)
    worst_r = worst_g = 0.0
    n_disk = 0
    for idx, (r, out) in sorted(res["kept"].items()):
        cam = r.bundle.camera(relsim.PRECISION_FP64)
        pix = rng.choice(r.rays, min(r.rays, 500), replace=False)
        ref = O.trace(relsim.camera_dict(cam), pixels=pix.astype(np.uint64), threads=0)
        st = out["status"][pix].astype(np.uint32)
        band = O.boundary_band(ref, O.lib().orc_isco_radius(1.0, cam.metric_spin), cam.disk_outer_radius, 1e-6)
        assert not ((st != ref["status"]) & ~band).any(), idx
        both = (st == O.DISK) & (ref["status"] == O.DISK)
        if both.any():
            n_disk += int(both.sum())
            worst_r = max(worst_r, float(np.max(np.abs(out["r_hit"][pix][both] - ref["r_hit"][both]) / ref["r_hit"][both])))
            worst_g = max(worst_g, float(np.max(np.abs(out["g"][pix][both] - ref["g"][both]) / ref["g"][both])))
    print(f"stream sample vs oracle: {n_disk} disk rays, r_hit rel max {worst_r:.2e}, g rel max {worst_g:.2e}")
    assert worst_r < 1e-5 and worst_g < 1e-5


def test_multi_source_request_matches_direct_trace(tracer):
    req = [r for r in scenes.request_stream() if r.multi_source][1]
    cam = req.bundle.camera(relsim.PRECISION_FP64)
    cam.screen_width = cam.screen_height = 64
    srcs = scenes.rt_sources(req.sources)
    with _server() as srv:
        a, out_a = srv.submit(cam, FIELDS, sources=srcs)
        b, out_b = srv.submit(config_cam("c2", width=64, height=64), FIELDS)  # mixed in with a single-hole one
        got = srv.wait([a, b])
    assert all(d.status == 0 for d in got.values())
    ref = tracer.dispatch_multi(cam, srcs, fields=list(FIELDS), pixels=False)
    for k in FIELDS:
        assert same(out_a[k], ref[k]), k


def test_shaded_requests_match_shaded_dispatch(tracer):
    """With rt_server_set_shading, a finished single-hole request's pixels are
    shaded (disk colour, tonemapping) at the first disk crossing -- the
    server's epochs hold no translucent-disk continuation -- as the shading
    oracle shades the request's own record, within 1e-6 sRGB; the rest of each
    pixel equals an unshaded rt_dispatch of the same camera; a multi-source
    request keeps black pixels; a server that does not record the fields the
    shading reads refuses it."""
    from test_gpu_shading import oracle_pixels

    sh = relsim.shading(tonemapping_mode=1, hydro_model=1)
    cams = [config_cam("c2", width=128, height=96, precision=relsim.PRECISION_MIXED),
            relsim.make_camera(spin=0.9, r_obs=50.0, incl_deg=75.0, fov_deg=30.0, width=96, height=64,
                               metric_form=relsim.METRIC_BOYER_LINDQUIST, charge=0.3)]
    tracer.set_launch_config()
    ref = [tracer.dispatch(c, fields=list(FIELDS), pixels=True) for c in cams]
    req = [r for r in scenes.request_stream() if r.multi_source][0]
    mcam = req.bundle.camera(relsim.PRECISION_FP64)
    mcam.screen_width = mcam.screen_height = 32
    with _server() as srv:
        srv.set_shading(sh)
        subs = [srv.submit(c, FIELDS, pixels=True) for c in cams]
        mid, mout = srv.submit(mcam, FIELDS, pixels=True, sources=scenes.rt_sources(req.sources))
        done = srv.wait([i for i, _ in subs] + [mid])
    for (rid, out), r, c in zip(subs, ref, cams):
        assert done[rid].status == relsim.RT_OK
        for f in ("status", "r_hit", "phi", "g"):
            assert np.array_equal(out[f], r[f], equal_nan=(out[f].dtype.kind == "f")), f
        want = oracle_pixels(c, sh, out["status"], out["r_hit"], out["phi"], out["g"])
        rgb = np.stack([out["pixels"]["r"], out["pixels"]["g"], out["pixels"]["b"]], 1)
        assert np.abs(rgb - want).max() < 1e-6
        for f in ("a", "redshift", "affine_parameter", "status_flags", "iterations_used"):
            assert np.array_equal(out["pixels"][f], r["pixels"][f]), f
        assert out["pixels"]["r"].max() > 0.0
    assert done[mid].status == relsim.RT_OK
    assert np.all(mout["pixels"]["r"] == 0.0) and np.all(mout["pixels"]["a"] == 1.0)
    with relsim.Server(0, relsim.server_config(1 << 26, record=("status", "pixels"))) as bare:
        with pytest.raises(relsim.RelsimError):
            bare.set_shading(sh)


def test_epochs_budgeted_by_cost(tracer):
    """Epochs are budgeted in cost units (a mixed ray 1, FP64 2, Boyer-Lindquist
    4, multi-source 4 per hole at rtol 1e-10 and 2 at the mixed mode's 1e-8),
    fill up to min_epoch_rays rays past that
    budget, and never hold more rays than epoch_rays, even when a row does not
    fit the room left (it waits for the next epoch); a row wider than an epoch
    is refused."""
    tracer.set_launch_config()
    cams = [config_cam("c2", width=96, height=40, precision=relsim.PRECISION_MIXED),
            config_cam("c2", width=100, height=30, precision=relsim.PRECISION_MIXED),
            config_cam("c3", width=70, height=20)]
    with _server(epoch_rays=1000, chunk_rays=1000) as srv:
        subs = [srv.submit(c, FIELDS) for c in cams]
        got = srv.wait([rid for rid, _ in subs])
        st = srv.stats()
        with pytest.raises(relsim.RelsimError) as e:
            srv.submit(config_cam("c2", width=1001, height=2), FIELDS)
        assert e.value.status == 1  # INVALID_ARG
    assert all(d.status == relsim.RT_OK for d in got.values())
    assert 0 < st.peak_epoch_rays <= 1000
    for cam, (rid, out) in zip(cams, subs):
        ref = tracer.dispatch(cam, fields=list(FIELDS), pixels=False)
        for k in FIELDS:
            assert same(out[k], ref[k]), k
    # a 4-hole FP64 scene costs 16 units a ray: 4096-unit epochs take 4 rows of 64
    req = [r for r in scenes.request_stream() if r.multi_source and len(r.sources) == 3][0]
    cam = req.bundle.camera(relsim.PRECISION_FP64)
    cam.screen_width = cam.screen_height = 64
    srcs = scenes.rt_sources(req.sources)
    ref = tracer.dispatch_multi(cam, srcs, fields=list(FIELDS), pixels=False)
    for floor, peak, epochs in ((1, 4 * 64, 16), (4096, 4096, 1)):
        with _server(epoch_rays=4096, chunk_rays=4096, min_epoch_rays=floor) as srv:
            rid, out = srv.submit(cam, FIELDS, sources=srcs)
            got = srv.wait([rid])
            st = srv.stats()
        assert got[rid].status == relsim.RT_OK
        assert (st.peak_epoch_rays, st.epochs) == (peak, epochs), floor
        for k in FIELDS:
            assert same(out[k], ref[k]), k


def test_exit_directions_are_refused():
    """The server does not record exit directions: a request asking for them is
    refused rather than left unwritten."""
    cam = config_cam("c2", width=32, height=32)
    with _server() as srv:
        with pytest.raises(relsim.RelsimError) as e:
            srv.submit(cam, FIELDS + ("exit_x",))
        assert e.value.status == 1
