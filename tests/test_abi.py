"""The C ABI library loads on the CPU, exports every entry point declared in
include/relsim_cuda.h, and its struct layouts match the header (compiled
here with gcc) and the ctypes mirror.  Host-only entry points run without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import relsim

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "relsim_cuda.h")


def declared_functions(path):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rt_[a-z_0-9]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    L = relsim.lib()
    names = declared_functions(HEADER)
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), name
    assert set(relsim.EXPORTS) <= set(names)


def test_layouts_match_header(tmp_path):
    prog = tmp_path / "sizes.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "relsim_cuda.h"\nint main(void){'
                    'printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(rt_camera), sizeof(rt_pixel_out),'
                    ' sizeof(rt_ray_out), sizeof(rt_launch_config), sizeof(rt_stats),'
                    ' offsetof(rt_camera, screen_width), offsetof(rt_camera, metric_form),'
                    ' offsetof(rt_camera, metric_charge), offsetof(rt_camera, mixed_critical_band),'
                    ' offsetof(rt_pixel_out, status_flags));'
                    'return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    exp = [ctypes.sizeof(relsim.Camera), ctypes.sizeof(relsim.PixelOut), ctypes.sizeof(relsim.RayOut),
           ctypes.sizeof(relsim.LaunchConfig), ctypes.sizeof(relsim.Stats),
           relsim.Camera.screen_width.offset, relsim.Camera.metric_form.offset, relsim.Camera.metric_charge.offset,
           relsim.Camera.mixed_critical_band.offset, relsim.PixelOut.status_flags.offset]
    assert got == exp
    assert got[1] == 32  # GpuPixelOutput (gpu_types.hpp:1111-1121)
    assert relsim.PIXEL_DTYPE.itemsize == 32


def test_shading_layout_matches_header(tmp_path):
    prog = tmp_path / "sh.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "relsim_cuda.h"\nint main(void){'
                    'printf("%zu %zu %zu %zu %zu\\n", sizeof(rt_shading), sizeof(rt_disk_profile),'
                    ' offsetof(rt_shading, disk_temperature_scale_k), offsetof(rt_shading, tonemapping_mode),'
                    ' offsetof(rt_disk_profile, edge_softness)); return 0;}\n')
    exe = tmp_path / "sh"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    exp = [ctypes.sizeof(relsim.Shading), ctypes.sizeof(relsim.DiskProfile),
           relsim.Shading.disk_temperature_scale_k.offset, relsim.Shading.tonemapping_mode.offset,
           relsim.DiskProfile.edge_softness.offset]
    assert got == exp
    assert got[1] == 128  # GpuDiskProfile (gpu_types.hpp:80 static_assert)
    s = relsim.shading()
    assert s.disk.peak_temperature_k == 9500.0 and s.disk_temperature_scale_k == 23796.0
    assert s.disk_doppler_beaming_exponent == 5.32 and s.sky_enabled == 0


def test_server_layouts_match_header(tmp_path):
    prog = tmp_path / "srv.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "relsim_cuda.h"\nint main(void){'
                    'printf("%zu %zu %zu %zu %zu\\n", sizeof(rt_server_config), sizeof(rt_request_done),'
                    ' sizeof(rt_server_stats), offsetof(rt_server_config, launch_mixed),'
                    ' offsetof(rt_request_done, status)); return 0;}\n')
    exe = tmp_path / "srv"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    exp = [ctypes.sizeof(relsim.ServerConfig), ctypes.sizeof(relsim.RequestDone), ctypes.sizeof(relsim.ServerStats),
           relsim.ServerConfig.launch_mixed.offset, relsim.RequestDone.status.offset]
    assert got == exp


def test_server_config_defaults_and_no_device():
    c = relsim.server_config()
    assert c.memory_budget_bytes == 1 << 30 and c.chunk_rays == 1 << 18 and c.epoch_rays == 1 << 22
    assert c.record_mask == sum(relsim.RECORD_BIT[f] for f in ("status", "r", "theta", "phi", "r_hit", "g", "pixels"))
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(relsim.RelsimError) as e:
        relsim.Server(0, c)
    assert e.value.status == 4  # DEVICE: no CPU fallback


def test_host_only_entry_points():
    L = relsim.lib()
    assert L.rt_abi_version() == 5
    c = relsim.Camera()
    L.rt_camera_defaults(ctypes.byref(c))
    assert c.screen_width == 2048 and c.metric_spin == 0.94 and c.rtol == 1e-10 and c.mixed_critical_band == 0.0
    # the default camera looks at the hole from r=100, 17 deg: forward = -e_r
    th = np.radians(17.0)
    np.testing.assert_allclose(list(c.tetrad_e1)[1:], [-np.sin(th), 0.0, -np.cos(th)], atol=1e-15)
    mine = relsim.make_camera()
    for f in ("tetrad_e1", "tetrad_e2", "tetrad_e3", "observer_position"):
        np.testing.assert_allclose(list(getattr(mine, f)), list(getattr(c, f)), atol=1e-15)
    cams = [relsim.make_camera(width=64, height=32), relsim.make_camera(width=10, height=10, row_offset=4, row_count=3),
            relsim.make_camera(width=10, height=10, row_offset=8, row_count=0)]
    assert relsim.bundle_rays(cams) == 64 * 32 + 30 + 20


def test_no_device_is_reported_not_hidden():
    """Without a GPU the library fails loudly (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    assert relsim.lib().rt_is_platform_supported() == 0
    with pytest.raises(relsim.RelsimError):
        relsim.Tracer(0)


def test_bench_descriptor_byte_counts(tmp_path):
    """bench.py's host-to-device bytes per image are the descriptors' sizes."""
    import shutil
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    prog = tmp_path / "sz.cu"
    prog.write_text('#include <cstdio>\n#include "rt_internal.h"\nint main(){ std::printf("%zu %zu %zu\\n", '
                    'sizeof(relsim::BundleDesc), sizeof(relsim::BlDesc), sizeof(relsim::ShadeDesc)); }\n')
    exe = tmp_path / "sz"
    subprocess.run([nvcc, "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", os.path.join(ROOT, "include"), "-I",
                    os.path.join(ROOT, "relativity-simulator_b200", "csrc"), str(prog), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert got == [bench.H2D_BYTES_PER_IMAGE, bench.BL_H2D_BYTES_PER_IMAGE, bench.SHADE_H2D_BYTES]
