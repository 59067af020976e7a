"""Edge cases of the Kerr-Schild tracers against the FP64 oracle (through the C ABI).

  - tiny and ragged images (1 x 1, single rows and columns, widths that are not
    a multiple of the warp size): same bars as the full images;
  - the attempt limit: rays that run out of attempts end UNFINISHED with the
    MAX_STEPS flag after the same attempts as on the oracle, at the same point
    within 1e-7 (the point is the last step boundary, not an event: the PI
    controller's FP32 log2/exp2 differ from the host's in the last ulp, which
    moves step boundaries by ~1e-7 of a step; terminal events are interpolated
    and meet the 1e-9 bar);
  - parameters at their clamps (spin beyond 0.999 M, an observer inside
    1.02 r_+, a negative spin), which both sides clamp the same way;
  - the largest image of this suite, 8192^2 = 67 M rays in one mixed-precision
    device dispatch: every ray classified, a sample within the mixed bars;
  - empty images are refused (INVALID_ARG) by the handle and by the server;
  - a host wait with a wall-clock limit returns TIMEOUT while work runs and the
    handle stays usable (failure detection without a GPU fault).
"""
import numpy as np
import pytest

import relsim
from cameras import config_cam
from oracle import oracle as O
from test_gpu_parity import _compare

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h", [(1, 1), (37, 1), (1, 37), (33, 31), (100, 3)])
def test_tiny_and_ragged_images(tracer, w, h):
    tracer.set_launch_config()
    cam = config_cam("c2", width=w, height=h, fov_deg=4.0)
    out, ref = _compare(tracer, cam)
    assert out["status"].size == w * h


def test_attempt_limit(tracer):
    tracer.set_launch_config()
    cam = config_cam("c3", width=48, height=48, max_steps=40)
    out = tracer.dispatch(cam)
    ref = O.trace(relsim.camera_dict(cam))
    unf = out["status"] == relsim.RAY_UNFINISHED
    assert unf.sum() > 100
    np.testing.assert_array_equal(out["status"], ref["status"])
    assert np.all(out["flags"][unf] & relsim.RAYFLAG_MAX_STEPS)
    assert np.all(ref["flags"][unf] & relsim.RAYFLAG_MAX_STEPS)
    assert np.all(out["steps_accepted"][unf] + out["steps_rejected"][unf] == 40)
    np.testing.assert_array_equal(out["steps_accepted"], ref["steps_accepted"])
    for f in ("r", "theta"):
        rel = np.abs(out[f][unf] - ref[f][unf]) / np.abs(ref[f][unf])
        assert rel.max() < 1e-7, (f, rel.max())
    assert np.max(np.abs(out["phi"][unf] - ref["phi"][unf])) < 1e-7
    # the rays that finished within the limit meet the usual bars
    fin = ~unf
    if fin.any():
        rel = np.abs(out["r"][fin] - ref["r"][fin]) / ref["r"][fin]
        assert rel.max() < 1e-9


@pytest.mark.parametrize("kw", [dict(spin=0.99995), dict(spin=-0.97, incl_deg=120.0),
                                dict(r_obs=1.5, spin=0.5, fov_deg=60.0), dict(r_obs=6.0, spin=0.9, fov_deg=90.0)])
def test_parameters_at_their_clamps(tracer, kw):
    tracer.set_launch_config()
    cam = relsim.make_camera(**{**dict(spin=0.94, r_obs=30.0, incl_deg=70.0, fov_deg=30.0, width=40, height=40), **kw})
    _compare(tracer, cam)


def test_largest_image_mixed(tracer):
    side = 8192
    n = side * side
    cam = config_cam("c2", width=side, height=side, precision=relsim.PRECISION_MIXED)
    tracer.set_launch_config()
    ro, dev = relsim.device_ray_out(n, ["status", "r_hit", "g"])
    tracer.dispatch_device(cam, ro, None, n)
    tracer.synchronize()  # the device entry point only enqueues
    st = dev["status"].cpu().numpy().view(np.uint32)
    counts = np.bincount(st, minlength=4)
    assert counts[relsim.RAY_UNFINISHED] == 0 and counts.sum() == n
    assert counts[relsim.RAY_DISK] > n // 2 and counts[relsim.RAY_CAPTURED] > 0
    rng = np.random.default_rng(11)
    pix = np.sort(rng.choice(n, 600, replace=False))
    ref = O.trace(relsim.camera_dict(config_cam("c2", width=side, height=side)), pixels=pix.astype(np.uint64))
    r_hit = dev["r_hit"].cpu().numpy()[pix]
    g = dev["g"].cpu().numpy()[pix]
    s = st[pix]
    band = O.boundary_band(ref, O.lib().orc_isco_radius(1.0, cam.metric_spin), cam.disk_outer_radius, 1e-6)
    assert not ((s != ref["status"]) & ~band).any()
    both = (s == O.DISK) & (ref["status"] == O.DISK)
    assert np.max(np.abs(r_hit[both] - ref["r_hit"][both]) / ref["r_hit"][both]) < 1e-6
    assert np.max(np.abs(g[both] - ref["g"][both]) / ref["g"][both]) < 1e-6


def test_empty_images_are_refused(tracer):
    for w, h in ((0, 16), (16, 0)):
        cam = config_cam("c2", width=w, height=h)
        with pytest.raises(relsim.RelsimError) as e:
            tracer.dispatch(cam, fields=["status"], pixels=True)
        assert e.value.status == 1  # INVALID_ARG
        with relsim.Server(0, relsim.server_config(1 << 24, record=("status",))) as srv:
            with pytest.raises(relsim.RelsimError) as e:
                srv.submit(cam, ("status",))
            assert e.value.status == 1
    assert tracer.is_ready()


def test_host_wait_times_out_and_recovers(tracer):
    """rt_synchronize with a wall-clock limit returns RT_ERR_TIMEOUT while a long
    trace is still running (the work is not cancelled and the handle stays
    usable); a wait without a limit then completes, and the records equal a
    host dispatch of the same camera."""
    side = 4096
    n = side * side
    cam = config_cam("c3", width=side, height=side)
    tracer.set_launch_config()
    ro, dev = relsim.device_ray_out(n, ["status", "r_hit"])
    tracer.dispatch_device(cam, ro, None, n)
    assert tracer.lib.rt_synchronize(tracer._h, 1.0) == 3  # TIMEOUT: about 0.2 s of work was enqueued
    assert tracer.is_ready()
    tracer.synchronize()
    st = dev["status"].cpu().numpy().view(np.uint32)
    assert np.all(st != relsim.RAY_UNFINISHED)
    small = config_cam("c3", width=side, height=side, row_offset=2000, row_count=8)
    part = tracer.dispatch(small, fields=["status", "r_hit"], pixels=False)
    np.testing.assert_array_equal(part["status"], st[2000 * side:2008 * side])
    np.testing.assert_array_equal(part["r_hit"], dev["r_hit"].cpu().numpy()[2000 * side:2008 * side])
