"""Allocation-free bundle trace, rt_trace_bundles_noalloc, through the C ABI.

The entry point keeps the persistent launch's scratch (ray-queue counter,
launch counters, bundle table) in a static device array instead of
handle-owned buffers.  Two calls in a row must each reproduce
rt_trace_bundles_device on the same bundle table (every call clears the
counters that must start at zero), repeated calls must leave the device's free
memory unchanged, and a bundle table longer than the static scratch holds is
rejected with a message before any device work.  The call cannot be captured
into a CUDA graph (it uploads the bundle table from its own stack frame), so on
a capturing stream it is refused before anything is enqueued.

This file is collected last so that it also runs after every other GPU test.
"""
import ctypes

import numpy as np
import pytest

import relsim
from cameras import config_cam

FIELDS = [name for name, _ in relsim.RAY_FIELDS]  # every record field, the drifts and exit directions too
FLOAT_FIELDS = [name for name, dt in relsim.RAY_FIELDS if dt == np.float64]
REL = 1e-12  # same kernel, same inputs: the records agree to rounding of the last digit at most


def _cams(precision):
    return [config_cam("c2", width=64, height=48, precision=precision),
            config_cam("c3", width=40, height=40, precision=precision),
            config_cam("c1", width=32, height=32, row_offset=8, row_count=16, precision=precision)]


def _outputs(n):
    import torch
    ro, t = relsim.device_ray_out(n, FIELDS)
    pix = torch.zeros(n * 32, dtype=torch.uint8, device="cuda")
    return ro, t, pix


def _host(t, pix):
    import torch
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in t.items()}
    out["pixels"] = pix.cpu().numpy()
    return out


def _assert_same(a, b):
    for k in ("status", "flags", "steps_accepted", "steps_rejected"):
        assert np.array_equal(a[k], b[k]), k
    for k in FLOAT_FIELDS:
        x, y = a[k], b[k]
        nan = np.isnan(y)
        assert np.array_equal(np.isnan(x), nan), k
        rel = np.abs(x[~nan] - y[~nan]) / np.maximum(np.abs(y[~nan]), 1e-300)
        assert rel.max(initial=0.0) <= REL, (k, rel.max())
    assert np.array_equal(a["pixels"], b["pixels"])


def test_noalloc_rejects_a_table_longer_than_its_scratch():
    """Host-side validation: no device is touched, so this runs without a GPU."""
    cams = [relsim.make_camera(width=4, height=4)] * (relsim.NOALLOC_MAX_BUNDLES + 1)
    ro = relsim.RayOut()
    with pytest.raises(relsim.RelsimError) as e:
        relsim.trace_bundles_noalloc(cams, ro, None, 16 * len(cams))
    assert e.value.status == 1 and "at most 32" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [relsim.PRECISION_FP64, relsim.PRECISION_MIXED])
def test_noalloc_matches_the_handle_entry_point_twice(precision):
    import torch
    cams = _cams(precision)
    n = relsim.bundle_rays(cams)
    with relsim.Tracer(0) as tr:
        # the allocation-free call runs the single-kernel tracer (no buffers for parked rays)
        tr.set_launch_config(mixed_single_kernel=1)
        ro, t, pix = _outputs(n)
        tr.trace_bundles_device(cams, ro, pix.data_ptr(), n)
        ref = _host(t, pix)
    assert np.all(ref["status"] != relsim.RAY_UNFINISHED)
    for _call in range(2):
        ro, t, pix = _outputs(n)
        relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n)
        _assert_same(_host(t, pix), ref)
    # explicit offsets (bundles written in reverse order) and an explicit launch shape
    sizes = [relsim.window_rays(c) for c in cams]
    offs = np.cumsum([0] + sizes[::-1][:-1])[::-1].astype(np.uint64)
    ro, t, pix = _outputs(n)
    relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n, offsets=offs,
                                 launch=relsim.LaunchConfig(128, 0, 32, 1, 0))
    got = _host(t, pix)
    begin = 0
    for size, off in zip(sizes, offs):
        part = {k: v[int(off):int(off) + size] for k, v in got.items() if k != "pixels"}
        part["pixels"] = got["pixels"].reshape(-1, 32)[int(off):int(off) + size].reshape(-1)
        want = {k: v[begin:begin + size] for k, v in ref.items() if k != "pixels"}
        want["pixels"] = ref["pixels"].reshape(-1, 32)[begin:begin + size].reshape(-1)
        _assert_same(part, want)
        begin += size
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_noalloc_leaves_device_memory_unchanged():
    import torch
    cams = _cams(relsim.PRECISION_FP64)
    n = relsim.bundle_rays(cams)
    ro, t, pix = _outputs(n)
    stream = torch.cuda.Stream()
    relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n, stream=stream.cuda_stream)  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.all(t["status"].cpu().numpy() != relsim.RAY_UNFINISHED)


@pytest.mark.gpu
def test_noalloc_reports_bad_arguments():
    cams = _cams(relsim.PRECISION_FP64)
    n = relsim.bundle_rays(cams)
    ro, t, pix = _outputs(n)
    with pytest.raises(relsim.RelsimError, match="capacity"):
        relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n - 1)
    with pytest.raises(relsim.RelsimError, match="one precision mode"):
        mixed = config_cam("c2", width=8, height=8, precision=relsim.PRECISION_MIXED)
        relsim.trace_bundles_noalloc(cams + [mixed], ro, pix.data_ptr(), n + 64)
    with pytest.raises(relsim.RelsimError, match="no such device"):
        relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n, device=1 << 20)
    with pytest.raises(relsim.RelsimError, match="16-byte"):
        relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr() + 4, n)


@pytest.mark.gpu
def test_noalloc_refuses_stream_capture():
    """A capturing stream is refused before anything is enqueued: the capture
    stays valid (it ends as an empty graph) and the caller's current device is
    unchanged."""
    import torch
    cams = _cams(relsim.PRECISION_FP64)
    n = relsim.bundle_rays(cams)
    ro, t, pix = _outputs(n)
    relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n)  # set-up call outside the capture
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        with pytest.raises(relsim.RelsimError, match="capturing") as e:
            relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n, stream=stream.cuda_stream)
    assert e.value.status == 1
    assert torch.cuda.current_device() == 0
    # the entry point still works on an ordinary stream afterwards
    relsim.trace_bundles_noalloc(cams, ro, pix.data_ptr(), n, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    assert np.all(t["status"].cpu().numpy() != relsim.RAY_UNFINISHED)
