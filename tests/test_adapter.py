"""The C++ adapter with VulkanComputeExecutor's method names
(include/relsim_executor.hpp), compiled with g++ against the C ABI library.

CPU: the push-constant mapping (spin clamp to 0.999 M, disk inner radius =
inner_radius_scale x r_ISCO, outer = outer_radius_mass_units x M), the answers
without a device (unsupported platform, initialise fails, dispatch returns
false: no CPU fallback), and, where the reference headers are present here,
that the mapping compiles against the reference's own GpuCameraPushConstants.
GPU: dispatch_and_readback gives the same pixels as rt_dispatch through the
Python binding, and a raised cancel flag makes it return false.
"""
import os
import subprocess

import numpy as np
import pytest

import relsim

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "adapter_main.cpp")
LIBDIR = os.path.dirname(relsim.LIB_PATH)
# the reference source tree, as oracle/Makefile takes it (REF_ROOT)
REFERENCE_INCLUDE = os.path.join(os.environ.get("REF_ROOT", "/root/reference"), "include")


def _build(tmp_path, extra=()):
    exe = tmp_path / "adapter_main"
    cmd = ["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), *extra, SRC, "-o", str(exe),
           "-L", LIBDIR, "-lrelsim_cuda", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return str(exe)


def test_push_constant_mapping(tmp_path):
    out = subprocess.run([_build(tmp_path), "map"], capture_output=True, text=True, check=True).stdout.split()
    spin, inner, outer, esc, w, h, steps, isco = (float(v) for v in out)
    assert spin == pytest.approx(0.999, abs=1e-15)
    assert inner == pytest.approx(1.5 * isco, rel=1e-15) and outer == 20.0 and esc == 1000.0
    assert (w, h, steps) == (96, 64, 20000)
    assert isco == pytest.approx(relsim.lib().rt_kerr_isco_radius(1.0, 0.999), rel=0)


def test_metric_type_routing(tmp_path):
    """Types 2/3 trace the Kerr-Schild form; 5 the Boyer-Lindquist Kerr-Newman
    form with the push constants' charge; 1 Boyer-Lindquist with spin and
    charge 0 (trace_exact_photon_dispatch, software_compute_engine.hpp:3316-3392)."""
    lines = subprocess.run([_build(tmp_path), "route"], capture_output=True, text=True, check=True).stdout.splitlines()
    rows = [ln.split() for ln in lines]
    assert rows[0] == ["3", "1", str(relsim.METRIC_KERR_SCHILD), "0.93999999999999995", "0"]
    assert rows[1] == ["5", "1", str(relsim.METRIC_BOYER_LINDQUIST), "0.93999999999999995", "0.40000000000000002"]
    assert rows[2] == ["1", "1", str(relsim.METRIC_BOYER_LINDQUIST), "0", "0"]
    assert rows[3] == ["0", "0"]


def test_shading_mapping(tmp_path):
    """The push constants' disk profile, overrides, time, exposure, tonemapping,
    hydro model with its torus settings and procedural sky (the GpuSkyProfile
    image) become rt_shading, with the sky drawn."""
    out = subprocess.run([_build(tmp_path), "shade"], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["7", "15000", "3", "2.5", "-1", "1", "1", "2", "1", "1", "6", "11", "1.33333", "0.35", "3"]


@pytest.mark.skipif(not os.path.isdir(REFERENCE_INCLUDE), reason="reference headers not present")
def test_shading_mapping_compiles_against_reference_push_constants(tmp_path):
    exe = _build(tmp_path, extra=("-std=c++23", "-DRELSIM_WITH_REFERENCE_TYPES", "-I", REFERENCE_INCLUDE))
    out = subprocess.run([exe, "shade"], capture_output=True, text=True, check=True).stdout.split()
    assert out[:3] == ["7", "15000", "3"] and out[8] == "1"


def test_no_device_answers(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    out = subprocess.run([_build(tmp_path), "cpu"], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["0", "0", "0", "0"]


@pytest.mark.skipif(not os.path.isdir(REFERENCE_INCLUDE), reason="reference headers not present")
def test_mapping_compiles_against_reference_push_constants(tmp_path):
    exe = _build(tmp_path, extra=("-std=c++23", "-DRELSIM_WITH_REFERENCE_TYPES", "-I", REFERENCE_INCLUDE))
    out = subprocess.run([exe, "map"], capture_output=True, text=True, check=True).stdout.split()
    assert float(out[2]) == 20.0 and int(out[4]) == 96


@pytest.mark.gpu
def test_adapter_dispatch_equals_c_abi(tmp_path, tracer):
    exe = _build(tmp_path)
    dump = tmp_path / "pix.bin"
    res = subprocess.run([exe, "gpu", str(dump)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    n, cancelled_ok, ready = (int(v) for v in res.stdout.split())
    assert n == 96 * 64 and cancelled_ok == 1 and ready == 1
    got = np.fromfile(dump, dtype=relsim.PIXEL_DTYPE)
    cam = relsim.make_camera(width=96, height=64)
    tracer.set_launch_config()
    ref = tracer.dispatch(cam, fields=[], pixels=True)["pixels"]
    assert np.array_equal(got, ref)
