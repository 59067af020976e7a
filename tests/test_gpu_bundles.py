"""Batched camera bundles in one persistent, graph-captured launch
(rt_trace_bundles_device) on the 512-bundle table (seed 0, about 97 M rays,
mixed precision).

  - every bundle's records equal a trace of that bundle alone (bundle sizes
    are multiples of 32 rays, so each warp's ray group and hence the mixed
    mode's precision choice is the same in both runs): bit-identical;
  - sampled rays of several bundles against the FP64 oracle at the mixed
    mode's stated error: class identical outside the 1e-6 M band, disk radius
    and g within 1e-5 relative (the table spans a up to 0.998 M and observers
    down to 20 M);
  - the captured graph replays the current bundle table's contents.
"""
import numpy as np
import pytest

import relsim
import scenes
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ["status", "steps_accepted", "steps_rejected", "phi", "r_hit", "g"]
SHAPE = (128, 0, 32, 1, 1)  # block, CTAs/SM (max), refill at 32 idle lanes, 1 ray per thread, rolled FP64


def same(a, b) -> bool:
    return np.array_equal(a, b, equal_nan=(a.dtype.kind == "f"))


@pytest.fixture(scope="module")
def c4(tracer):
    import torch
    cams = scenes.bundle_cameras(512, 0)
    n = relsim.bundle_rays(cams)
    ro, t = relsim.device_ray_out(n, FIELDS)
    tracer.set_launch_config(*SHAPE)
    tracer.trace_bundles_device(cams, ro, None, n)
    st = tracer.stats()
    out = {k: v.cpu().numpy() for k, v in t.items()}
    del t
    torch.cuda.empty_cache()
    begins = np.cumsum([0] + [c.screen_width * c.screen_height for c in cams])
    yield cams, out, begins, st
    tracer.set_launch_config()


def test_c4_table_is_traced_completely(c4):
    cams, out, begins, st = c4
    assert begins[-1] > 90_000_000
    assert st.rays == begins[-1]
    assert st.kernel_ms > 0.0
    assert np.all(out["status"] != relsim.RAY_UNFINISHED)


def test_c4_bundles_equal_alone(tracer, c4):
    cams, out, begins, _ = c4
    rng = np.random.default_rng(5)
    tracer.set_launch_config(*SHAPE)
    for b in rng.choice(len(cams), 12, replace=False):
        cam = cams[b]
        n = cam.screen_width * cam.screen_height
        ro, t = relsim.device_ray_out(n, FIELDS)
        tracer.dispatch_device(cam, ro, None, n)
        tracer.synchronize()
        for k in FIELDS:
            alone = t[k].cpu().numpy()
            mine = out[k][begins[b]:begins[b] + n]
            assert same(alone, mine), (b, k)


def test_c4_sample_against_fp64_oracle(c4):
    cams, out, begins, _ = c4
    rng = np.random.default_rng(9)
    worst_r, worst_g = 0.0, 0.0
    for b in rng.choice(len(cams), 8, replace=False):
        cam = cams[b]
        n = cam.screen_width * cam.screen_height
        pix = rng.choice(n, min(n, 150), replace=False)
        ref_cam = relsim.camera_dict(cam)
        ref_cam["precision_mode"] = relsim.PRECISION_FP64
        ref_cam["rtol"] = ref_cam["atol"] = 1e-10
        ref = O.trace(ref_cam, pixels=pix.astype(np.uint64))
        st = out["status"][begins[b] + pix].astype(np.uint32)
        r_in = O.lib().orc_isco_radius(1.0, cam.metric_spin)
        band = O.boundary_band(ref, r_in, cam.disk_outer_radius, 1e-6)
        assert not ((st != ref["status"]) & ~band).any(), b
        both = (st == O.DISK) & (ref["status"] == O.DISK)
        if both.any():
            rh = out["r_hit"][begins[b] + pix][both]
            g = out["g"][begins[b] + pix][both]
            worst_r = max(worst_r, float(np.max(np.abs(rh - ref["r_hit"][both]) / ref["r_hit"][both])))
            worst_g = max(worst_g, float(np.max(np.abs(g - ref["g"][both]) / ref["g"][both])))
    print(f"c4 sample: r_hit rel max {worst_r:.2e}, g rel max {worst_g:.2e}")
    assert worst_r < 1e-5 and worst_g < 1e-5, (worst_r, worst_g)


def test_graph_replays_new_table_contents(tracer):
    """Same table shape, different cameras: the replayed graph traces the new ones."""
    draws = scenes.bundle_table(6, 3)
    cams_a = [d.camera() for d in draws]
    cams_b = [relsim.make_camera(spin=0.5, r_obs=40.0 + 10 * i, incl_deg=30.0 + 5 * i, fov_deg=15.0,
                                 width=d.side, height=d.side, precision=relsim.PRECISION_MIXED)
              for i, d in enumerate(draws)]
    n = relsim.bundle_rays(cams_a)
    ro, t = relsim.device_ray_out(n, ["status", "r_hit", "g", "phi"])
    tracer.set_launch_config(*SHAPE)
    outs = []
    for cams in (cams_a, cams_b, cams_a):  # same shape: the second and third calls replay the graph
        tracer.trace_bundles_device(cams, ro, None, n)
        tracer.synchronize()  # the tracer's stream, not torch's
        outs.append({k: v.cpu().numpy() for k, v in t.items()})
    first, second, third = outs
    for k in first:
        assert same(first[k], third[k]), k
    assert not np.array_equal(first["phi"], second["phi"])
    begin = 0
    for cam in cams_b:
        m = cam.screen_width * cam.screen_height
        ro1, t1 = relsim.device_ray_out(m, ["status", "r_hit", "g", "phi"])
        tracer.dispatch_device(cam, ro1, None, m)
        tracer.synchronize()
        for k in ("status", "r_hit", "g", "phi"):
            assert same(t1[k].cpu().numpy(), second[k][begin:begin + m]), k
        begin += m
    tracer.set_launch_config()
