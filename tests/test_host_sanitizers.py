"""Host-side code under AddressSanitizer and UndefinedBehaviorSanitizer (CPU).

The library's per-camera table builders (csrc/rt_bundle.cpp) and the CPU
oracles are compiled with -fsanitize=address,undefined into a small harness
(tests/native/sanitize_main.cpp).  The harness covers cameras at and beyond
their clamps, one-pixel and ragged screens, row windows past the screen,
source tables with spins past the clamp and zero axes, and a few traced rays
of each oracle form.  Any sanitizer report aborts the run.  The device code
is not covered here: it is held to the oracle by the GPU parity tests.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SAN = ["-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer"]


def test_host_code_is_sanitizer_clean(tmp_path):
    if not shutil.which("gcc") or not shutil.which("g++"):
        pytest.skip("no host compiler")
    objs = []
    for name in ("ks_oracle", "ms_oracle", "bl_oracle", "shade_oracle"):
        obj = str(tmp_path / f"{name}.o")
        subprocess.run(["gcc", "-std=c11", *SAN, "-pthread", "-c", os.path.join(ROOT, "oracle", f"{name}.c"), "-o",
                        obj], check=True)
        objs.append(obj)
    exe = str(tmp_path / "sanitize_main")
    subprocess.run(["g++", "-std=c++17", *SAN, "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "relativity-simulator_b200", "csrc"), "-I", os.path.join(ROOT, "oracle"),
                    os.path.join(ROOT, "tests", "native", "sanitize_main.cpp"),
                    os.path.join(ROOT, "relativity-simulator_b200", "csrc", "rt_bundle.cpp"), *objs, "-lm",
                    "-lpthread", "-o", exe], check=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1", UBSAN_OPTIONS="print_stacktrace=1")
    res = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    assert res.stdout.strip().endswith("ok")
