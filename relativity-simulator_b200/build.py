"""Build the tracer's shared library for sm_100a (in-tree).

    python relativity-simulator_b200/build.py [--verbose]

Output: relativity-simulator_b200/librelsim_cuda.so, exporting the C ABI of
include/relsim_cuda.h.  Compiles for sm_100a only (`-gencode
arch=compute_100a,code=sm_100a`); nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "librelsim_cuda.so")
BUILD = os.path.join(HERE, "_build")

SOURCES = ["rt_trace.cu", "rt_multi.cu", "rt_bl.cu", "rt_shade.cu", "rt_api.cu", "rt_server.cu", "rt_peak.cu", "rt_bundle.cpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "relsim_cuda.h"))
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [path] + headers):
            continue
        cmd = [nvcc(), *common, *GENCODE, "-lineinfo", "-c", path, "-o", obj]
        if src.endswith(".cu") and verbose:
            cmd += ["-Xptxas", "-v"]
        if src.endswith(".cpp"):
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-I", INCLUDE, "-I", CSRC, "-c", path, "-o", obj]
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        subprocess.run([nvcc(), *GENCODE, "-shared", "-cudart", "static", "-o", LIB, *objs], check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
