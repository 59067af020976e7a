#!/usr/bin/env python
"""Benchmark of the B200 null-geodesic tracer on the headline workload.

Workload: Kerr a=0.94 M, 2048x2048 pinhole camera at r=100 M, inclination
17 deg, FOV 12 deg, thin disk [r_ISCO, 20 M], <= 20000 attempts per ray
(synthetic camera grid; no dataset).  A step = one trace of the whole image.
Two tracers are timed in one run: the plain FP64 tracer (DP45 rtol=atol=1e-10)
and the mixed-precision tracer (FP32 far-zone stages, rtol=atol=1e-8); the mixed
image is compared ray by ray with the FP64 image, which gives its stated error
(the FP64 tracer itself is held to the FP64 oracle by tests/test_gpu_parity.py).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision both|fp64|mixed]
  python bench.py --impl reference      # the reference's own CPU image path

value: Mrays/s of the mixed tracer (the fp64 one with --precision fp64) with
       outputs resident in HBM, tracer kernel timed with CUDA events on its
       stream, L2 flushed between steps (a 256 MiB write); "precisions" holds
       both tracers' numbers and "mixed_vs_fp64" their ratio.
serving: the seeded request stream (2000 requests, Poisson 200/s) replayed in
       real time through the continuous-batching server (N = 1): p50/p99
       request latency, throughput and the error of sampled requests.
e2e:   Mrays/s through rt_dispatch (the dispatch_and_readback-shaped C call)
       into pinned host pixels (32-byte GpuPixelOutput, what the reference's
       call returns), host<->device copies inside the timed region, pixels
       shaded (disk colour and tonemapping, rt_set_shading defaults); its
       per-image p50/p99 wall latency.  e2e.with_records: the same call that
       also copies back the per-ray records (class, r, theta, phi, r_hit, g).
N > 1: one independent image per GPU (replicas, no collective); value is the
       total over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "relativity-simulator_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Mrays/s on Kerr a=0.94 2048^2, mixed vs FP64 at stated error; p50/p99 latency"
FLOP_PER_ATTEMPT = 1578.0  # Kerr-Schild RHS as written (206 ops) x 6 + DP45 stage/error ops
SIDE = 2048
RECORD_FIELDS = ["status", "r", "theta", "phi", "r_hit", "g"]
H2D_BYTES_PER_IMAGE = 464  # one bundle descriptor (per-camera constants) per image
# Boyer-Lindquist Kerr-Newman path (metric type 5): the reference's RHS as written,
# KerrNewmanMetric::christoffel_symbols (88 ops of metric derivatives, 37 of the
# inverse metric, 240 of the lambda loop over its 6 non-zero entries) and the
# RK45 contraction -Gamma u u (144 ops) = 509 ops, x 6 evaluations, + 488 ops of
# stage sums and error norm for the reference's 8-component state
BL_FLOP_PER_ATTEMPT = 3542.0
# kernels one device-resident trace of the image launches: the two-pass mixed
# tracer runs 4 rounds of a far and a near pass and one finish pass (the
# library's round count); the single-kernel tracers launch once
MIXED_TWO_PASS_LAUNCHES = 2 * 4 + 1
BL_CAMERA = dict(spin=0.9, charge=0.3, r_obs=50.0, incl_deg=75.0, fov_deg=30.0)
BL_H2D_BYTES_PER_IMAGE = 352  # the Boyer-Lindquist camera descriptor (sizeof BlDesc)
SHADE_H2D_BYTES = 3248  # the shading pass's per-camera constants with the sky profile and torus (sizeof ShadeDesc)
# what the e2e pixels hold: the reference's CPU dispatch shades every pixel the same way
# (its push-constant defaults have the procedural sky on)
PIXELS_NOTE = ("shaded: translucent disk (colour and opacity at every crossing), the default procedural sky "
               "behind rays that escape with throughput left, tonemapping")


def headline_camera(relsim, precision: int, side: int = SIDE):
    return relsim.make_camera(spin=0.94, r_obs=100.0, incl_deg=17.0, fov_deg=12.0, width=side, height=side,
                              precision=precision)


class ClockSampler:
    """SM clock, power and clock-event reasons sampled through NVML every 10 ms
    during the timed region (read-only queries; nvidia-smi at 200 ms when the
    NVML bindings are missing)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []  # (sm_mhz, max_mhz, power_w, util_pct, reason_bits)
        self.stop = None
        self.thread = None
        self.proc = None
        self.path = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.gpu)
        for get in (lambda: pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(p.uuid)),
                    lambda: pynvml.nvmlDeviceGetHandleByPciBusId(
                        f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"),
                    lambda: pynvml.nvmlDeviceGetHandleByIndex(self.gpu)):
            try:
                return pynvml, get()
            except Exception:
                continue
        raise RuntimeError("no NVML handle")

    def _poll(self, nv, h):
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx,
                                  nv.nvmlDeviceGetPowerUsage(h) / 1e3, nv.nvmlDeviceGetUtilizationRates(h).gpu,
                                  nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception:
                break
            self.stop.wait(0.01)

    def __enter__(self):
        import threading

        try:
            nv, h = self._nvml_handle()
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                     "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            except OSError:
                self.proc = None
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def _smi_rows(self):
        def num(v):
            try:
                return float(v)
            except ValueError:
                return float("nan")

        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 10:
                        bits = sum(b for i, b in enumerate(self.REASONS.values()) if parts[6 + i].lower() == "active")
                        rows.append((num(parts[1]), num(parts[2]), num(parts[3]), num(parts[4]), bits))
        except (OSError, TypeError):
            pass
        return rows

    def summary(self) -> dict:
        rows = self.rows if self.thread is not None else self._smi_rows()
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        load = [r for r in rows if r[3] > 50] or rows
        reasons = sorted({name for r in load for name, bit in self.REASONS.items() if int(r[4]) & bit})
        return {"sm_mhz": float(np.median([r[0] for r in load])), "sm_max_mhz": float(load[0][1]),
                "reasons": reasons, "samples": len(load), "power_w_max": float(max(r[2] for r in load)),
                "source": "NVML, 10 ms" if self.thread is not None else "nvidia-smi, 200 ms"}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_port_baseline(cam_dict: dict, seconds: float = 15.0) -> dict:
    """The FP64 oracle (same DP45 algorithm) on a random sample of the workload's rays, all host cores."""
    from oracle import oracle as O

    rng = np.random.default_rng(0)
    n_pix = cam_dict["screen_width"] * cam_dict["screen_height"]
    cores = os.cpu_count() or 1
    probe = rng.choice(n_pix, 2000, replace=False).astype(np.uint64)
    t0 = time.perf_counter()
    O.trace(cam_dict, pixels=probe, threads=cores)
    rate = probe.size / max(time.perf_counter() - t0, 1e-6)
    n = int(min(max(rate * seconds, 4000), n_pix))
    sample = rng.choice(n_pix, n, replace=False).astype(np.uint64)
    t0 = time.perf_counter()
    O.trace(cam_dict, pixels=sample, threads=cores)
    dt = time.perf_counter() - t0
    return {"value": n / dt / 1e6, "unit": "Mrays/s", "cores": cores, "kind": "port",
            "sample": f"{n} uniformly random rays of the 2048^2 image, FP64 DP45 oracle (oracle/ks_oracle.c), "
                      f"{dt:.1f} s"}


def reference_arm(args) -> None:
    """The reference's own CPU image path (SoftwareComputeEngine::dispatch_fp64, heuristic-step RK4,
    built from its headers into oracle/_ref) on row bands of the same camera."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    import relsim

    cam = headline_camera(relsim, relsim.PRECISION_FP64)
    d = relsim.camera_dict(cam)
    W = H = SIDE
    cores = os.cpu_count() or 1
    if not O.ref_available():
        try:
            O.build(ref=True)
        except Exception:
            pass
    if O.ref_available():
        R = O.ref()
        obs = np.ascontiguousarray(d["observer_position"], dtype=np.float64)
        e1 = np.ascontiguousarray(d["tetrad_e1"], dtype=np.float64)
        e2 = np.ascontiguousarray(d["tetrad_e2"], dtype=np.float64)
        e3 = np.ascontiguousarray(d["tetrad_e3"], dtype=np.float64)

        def image(side):
            st = np.zeros(side * side, np.uint32)
            it = np.zeros(side * side, np.uint32)
            z = np.zeros(side * side, np.float32)
            return R.ref_dispatch_fp64(O._p(obs), O._p(e1), O._p(e2), O._p(e3), d["field_of_view_rad"], 1.0, 0.94,
                                       1000.0, 20.0, side, side, 20000, 0, 0, O._p(st), O._p(it), O._p(z))
        kind = "reference"
        # sample: the same camera at a reduced resolution (a uniform grid over the same
        # field of view), whole images, so the reference's own split of the image
        # rows over hardware_concurrency threads applies; side chosen for ~6 s a step
        t = image(256)
        side = int(min(max(256 * math.sqrt(6.0 / max(t, 1e-3)) // 64 * 64, 256), SIDE))
        times = []
        for i in range(args.warmup + args.steps):
            dt = image(side)
            if i >= args.warmup:
                times.append(dt)
        n = side * side
        what = (f"SoftwareComputeEngine::dispatch_fp64 (reference image path, heuristic-step RK4) on the same "
                f"camera at {side}^2 (whole images), hardware_concurrency threads")
    else:
        kind = "port"
        what = "FP64 DP45 oracle (oracle/ks_oracle.c); the reference library was not built"
        rng = np.random.default_rng(1)
        n = 20000
        times = []
        for i in range(args.warmup + args.steps):
            pix = rng.choice(W * H, n, replace=False).astype(np.uint64)
            t0 = time.perf_counter()
            O.trace(d, pixels=pix, threads=cores)
            if i >= args.warmup:
                times.append(time.perf_counter() - t0)
    value = n * len(times) / sum(times) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "Kerr a=0.94 2048^2 pinhole r=100 i=17 FOV 12 disk [r_isco,20]",
                   "sample": f"{n} rays per step ({what})"},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": cores, "kind": kind,
                         "sample": f"{n} rays per step, {what}"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def time_device(tr, relsim, cam, n, ro, pix, flush, steps: int, warmup: int) -> dict:
    """K timed traces of the image into resident device outputs; L2 flushed before each."""
    import torch

    for _ in range(warmup):
        tr.dispatch_device(cam, ro, pix.data_ptr(), n)
        tr.stats()
    torch.cuda.synchronize()
    ms, attempts, accepted, rhs, fp64_att = [], 0, 0, 0, 0
    for _ in range(steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        tr.dispatch_device(cam, ro, pix.data_ptr(), n)
        s = tr.stats()  # waits; kernel_ms from events on the tracer's stream
        ms.append(s.kernel_ms)
        attempts += s.attempts
        accepted += s.accepted
        rhs += s.rhs_evals
        fp64_att += s.fp64_attempts
    return {"ms": ms, "attempts": attempts, "accepted": accepted, "rhs": rhs, "fp64_attempts": fp64_att}


def time_e2e(tr, relsim, cam, n, steps: int, warmup: int, fields=()):
    """Trace and shade (translucent disk, default procedural sky, tonemapping) through
    rt_dispatch (host buffers, copies inside), as the reference's dispatch_and_readback
    returns coloured pixels (32-byte
    GpuPixelOutput), plus the per-ray record fields asked for; per-image wall latency."""
    import torch

    host = {f: torch.empty(n, dtype=(torch.int32 if f == "status" else torch.float64), pin_memory=True)
            for f in fields}
    hpix = torch.empty(n * 32, dtype=torch.uint8, pin_memory=True)
    hro = relsim.RayOut()
    for f, t in host.items():
        setattr(hro, f, t.data_ptr())
    L = relsim.lib()
    lat = []
    tr.set_shading(relsim.shading(sky_enabled=1))
    try:
        for i in range(warmup + steps):
            t0 = time.perf_counter()
            st = L.rt_dispatch(tr.handle, ctypes.byref(cam), hpix.data_ptr(), ctypes.byref(hro) if fields else None,
                               n, None)
            dt = time.perf_counter() - t0
            if st != 0:
                raise RuntimeError(L.rt_last_error(tr.handle).decode())
            if i >= warmup:
                lat.append(dt)
    finally:
        tr.set_shading(None)
    return host, lat


def record_bytes(fields) -> int:
    return sum(4 if f == "status" else 8 for f in fields)


def time_bundles(tr, relsim, steps: int, warmup: int, device: str) -> dict:
    """The 512-bundle table (seed 0, mixed precision) in one graph-captured persistent
    launch per step, outputs resident on the device; device time from the tracer's events."""
    import torch

    import scenes
    from autotune import apply_tuned

    cams = scenes.bundle_cameras(512, 0)
    n = relsim.bundle_rays(cams)
    ro, _t = relsim.device_ray_out(n, ["status", "r_hit", "g"], device=device)
    pix = torch.empty(n * 32, dtype=torch.uint8, device=device)
    apply_tuned(tr, "mixed")
    for _ in range(warmup):
        tr.trace_bundles_device(cams, ro, pix.data_ptr(), n)
        tr.stats()
    ms, attempts = [], 0
    for _ in range(steps):
        tr.trace_bundles_device(cams, ro, pix.data_ptr(), n)  # graph replay
        s = tr.stats()
        ms.append(s.kernel_ms)
        attempts += s.attempts
    del ro, _t, pix
    torch.cuda.empty_cache()
    return {"workload": "512 bundles, seed 0: side round32(logU[64,1024]), a U[0,0.998], i U[5,85] deg, "
                        "r_obs logU[20,500] M, FOV U[8,40] deg; mixed precision; one CUDA-graph launch per step",
            "rays_per_step": n, "value": n * steps / (sum(ms) * 1e-3) / 1e6, "unit": "Mrays/s",
            "ms_per_step": sum(ms) / steps, "attempts_per_ray": attempts / (n * steps),
            "launch": vars_of(tr.launch_config())}


def bl_camera(relsim, side: int):
    return relsim.make_camera(width=side, height=side, metric_form=relsim.METRIC_BOYER_LINDQUIST, **BL_CAMERA)


def time_boyer_lindquist(tr, relsim, side, ro, pix, flush, steps, warmup, fp64_peak, fp32_peak, ws, device) -> dict:
    """The Boyer-Lindquist Kerr-Newman tracer on its own workload: device time with
    resident outputs (L2 flushed between steps) and end to end through rt_dispatch."""
    cam = bl_camera(relsim, side)
    n = side * side
    tr.set_launch_config()
    d = time_device(tr, relsim, cam, n, ro, pix, flush, steps, warmup)
    own_ms = float(sum(d["ms"]))
    total_ms = max_over_ranks(own_ms, ws, device)
    _, lat = time_e2e(tr, relsim, cam, n, steps, warmup)
    e2e_wall = max_over_ranks(sum(lat), ws, device)
    _, lat_rec = time_e2e(tr, relsim, cam, n, steps, warmup, RECORD_FIELDS)
    rec_wall = max_over_ranks(sum(lat_rec), ws, device)
    achieved = d["attempts"] * BL_FLOP_PER_ATTEMPT / (own_ms * 1e-3) / 1e12
    return {
        "workload": f"Kerr-Newman a=0.9 Q=0.3 {side}^2 pinhole r=50 M i=75 deg FOV 30 deg, disk [r_isco, 20 M]; "
                    f"Boyer-Lindquist geodesic equation (-Gamma u u), ZAMO observer, FP64 DP45 rtol=atol=1e-10",
        "value": replica_value(n, ws, steps, total_ms), "unit": "Mrays/s", "ms_per_step": total_ms / steps,
        "attempts_per_ray": d["attempts"] / (n * steps), "msteps_per_s": d["accepted"] / (own_ms * 1e-3) / 1e6,
        "latency_ms": {"kernel_p50": float(np.percentile(d["ms"], 50)), "kernel_p99": float(np.percentile(d["ms"], 99)),
                       "e2e_p50": 1e3 * float(np.percentile(lat, 50)), "e2e_p99": 1e3 * float(np.percentile(lat, 99))},
        "e2e": {"value": replica_value(n, ws, steps, e2e_wall * 1e3), "unit": "Mrays/s",
                "h2d_bytes_per_step": BL_H2D_BYTES_PER_IMAGE + SHADE_H2D_BYTES, "d2h_bytes_per_step": n * 32,
                "pixels": PIXELS_NOTE,
                "with_records": {"value": replica_value(n, ws, steps, rec_wall * 1e3), "fields": RECORD_FIELDS,
                                 "d2h_bytes_per_step": n * (32 + record_bytes(RECORD_FIELDS))}},
        "roofline": {"bound": "fp64 pipe", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp64_peak, "flop_per_attempt": BL_FLOP_PER_ATTEMPT,
                     "peak_source": "measured in this run: register FMA-chain kernel (rt_measure_fma_peak)",
                     "traffic": committed_traffic("bl"),
                     "executed": executed_roofline("bl", d["attempts"], own_ms, fp64_peak, fp32_peak)},
    }


def bl_cpu_baselines(side: int, seconds: float) -> dict:
    """The reference's own CPU path for the same Kerr-Newman camera (trace_exact_photon,
    heuristic RK4, oracle/_ref) on whole images at a reduced side, and the FP64 DP45
    oracle (oracle/bl_oracle.c) on a random sample of the full image's rays."""
    from oracle import oracle as O
    import relsim

    cores = os.cpu_count() or 1
    out = {}
    d = relsim.camera_dict(bl_camera(relsim, side))
    if O.ref_available():
        R = O.ref()
        obs, e1, e2, e3 = (np.ascontiguousarray(d[k], dtype=np.float64)
                           for k in ("observer_position", "tetrad_e1", "tetrad_e2", "tetrad_e3"))

        def image(w):
            st = np.zeros(w * w, np.uint32)
            it = np.zeros(w * w, np.uint32)
            z = np.zeros(w * w, np.float32)
            t = R.ref_dispatch_fp64_kn(O._p(obs), O._p(e1), O._p(e2), O._p(e3), d["field_of_view_rad"], 1.0,
                                       BL_CAMERA["spin"], BL_CAMERA["charge"], 1000.0, 20.0, w, w, 20000, 0, 0, 1.0,
                                       O._p(st), O._p(it), O._p(z))
            return t, float(it.mean())
        t, _ = image(64)
        w = int(min(max(64 * math.sqrt(seconds / 2 / max(t, 1e-3)) // 32 * 32, 64), side))
        t, iters = image(w)
        out["reference"] = {"value": w * w / t / 1e6, "unit": "Mrays/s", "cores": cores, "kind": "reference",
                            "sample": f"SoftwareComputeEngine::dispatch_fp64 (metric type 5, trace_exact_photon, "
                                      f"heuristic-step RK4, {iters:.1f} steps/ray) on the same camera at {w}^2, "
                                      f"hardware_concurrency threads, {t:.1f} s"}
    rng = np.random.default_rng(0)
    probe = rng.choice(side * side, 500, replace=False).astype(np.uint64)
    t0 = time.perf_counter()
    O.bl_trace(d, BL_CAMERA["charge"], pixels=probe, threads=cores)
    rate = probe.size / max(time.perf_counter() - t0, 1e-6)
    n = int(min(max(rate * seconds / 2, 2000), side * side))
    sample = rng.choice(side * side, n, replace=False).astype(np.uint64)
    t0 = time.perf_counter()
    O.bl_trace(d, BL_CAMERA["charge"], pixels=sample, threads=cores)
    dt = time.perf_counter() - t0
    out["port"] = {"value": n / dt / 1e6, "unit": "Mrays/s", "cores": cores, "kind": "port",
                   "sample": f"{n} uniformly random rays of the {side}^2 image, FP64 DP45 oracle (oracle/bl_oracle.c), "
                             f"{dt:.1f} s"}
    return out


def max_over_ranks(x: float, ws: int, device: str) -> float:
    """The slowest rank's time (every rank gets it); one all-reduce, no data-path collective."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(rays_per_rank: int, ws: int, steps: int, slowest_ms: float) -> float:
    """Whole-job Mrays/s of N independent replicas: all ranks' rays over the slowest rank's time."""
    return ws * rays_per_rank * steps / (slowest_ms * 1e-3) / 1e6


def ours(args) -> None:
    import torch

    import relsim

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from autotune import apply_tuned

    tr = relsim.Tracer(local)
    fp64_peak, fp32_peak = tr.measure_fma_peak()
    n = args.side * args.side
    ro, tensors = relsim.device_ray_out(n, RECORD_FIELDS, device=f"cuda:{local}")
    pix = torch.empty(n * 32, dtype=torch.uint8, device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    precisions = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    headline = precisions[-1]  # the mixed tracer when both run

    res = {}
    with ClockSampler(local) as clk:
        for prec in precisions:
            code = relsim.PRECISION_MIXED if prec == "mixed" else relsim.PRECISION_FP64
            cam = headline_camera(relsim, code, args.side)
            apply_tuned(tr, prec)
            if ws > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            wall0 = time.perf_counter()
            d = time_device(tr, relsim, cam, n, ro, pix, flush, args.steps, args.warmup)
            torch.cuda.synchronize()
            d["wall_s"] = time.perf_counter() - wall0
            d["cam"] = cam
            d["launch"] = vars_of(tr.launch_config())
            res[prec] = d
    clocks = clk.summary()

    # end to end through rt_dispatch (host buffers) for the headline precision
    hcam = res[headline]["cam"]
    apply_tuned(tr, headline)
    _, lat = time_e2e(tr, relsim, hcam, n, args.steps, args.warmup)
    e2e_wall = max_over_ranks(sum(lat), ws, f"cuda:{local}")
    e2e_value = replica_value(n, ws, args.steps, e2e_wall * 1e3)
    d2h = n * 32
    _, lat_rec = time_e2e(tr, relsim, hcam, n, args.steps, args.warmup, RECORD_FIELDS)
    rec_wall = max_over_ranks(sum(lat_rec), ws, f"cuda:{local}")
    e2e_records = {"value": replica_value(n, ws, args.steps, rec_wall * 1e3), "fields": RECORD_FIELDS,
                   "d2h_bytes_per_step": n * (32 + record_bytes(RECORD_FIELDS)),
                   "latency_ms_p50": 1e3 * float(np.percentile(lat_rec, 50)),
                   "latency_ms_p99": 1e3 * float(np.percentile(lat_rec, 99))}

    batched = None
    if not args.no_bundles:
        batched = time_bundles(tr, relsim, args.steps, args.warmup, f"cuda:{local}")

    bl = None
    if not args.no_bl:
        bl = time_boyer_lindquist(tr, relsim, args.side, ro, pix, flush, args.steps, args.warmup, fp64_peak, fp32_peak,
                                  ws, f"cuda:{local}")
        if rank == 0 and ws == 1 and not args.no_cpu_baseline:
            bl["cpu_baseline"] = bl_cpu_baselines(args.side, args.cpu_seconds)

    summary = {}
    for prec, d in res.items():
        own_ms = float(sum(d["ms"]))
        total_ms = max_over_ranks(own_ms, ws, f"cuda:{local}")
        peak = fp64_peak if prec == "fp64" else fp32_peak
        achieved = d["attempts"] * FLOP_PER_ATTEMPT / (own_ms * 1e-3) / 1e12
        summary[prec] = {
            "value": replica_value(n, ws, args.steps, total_ms), "ms_per_step": total_ms / args.steps,
            "p50_ms": float(np.percentile(d["ms"], 50)), "p99_ms": float(np.percentile(d["ms"], 99)),
            "msteps_per_s": d["accepted"] / (own_ms * 1e-3) / 1e6,
            "attempts_per_ray": d["attempts"] / (n * args.steps),
            "fp64_attempt_share": d["fp64_attempts"] / max(d["attempts"], 1),
            "rtol": d["cam"].rtol, "launch": d["launch"],
            "roofline": {"bound": "fp64 pipe" if prec == "fp64" else "fp32 pipe (fp64 state and near zone)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": "measured in this run: register FMA-chain kernel (rt_measure_fma_peak)",
                         "flop_per_attempt": FLOP_PER_ATTEMPT,
                         "traffic": committed_traffic(prec),
                         "executed": executed_roofline(prec, d["attempts"], own_ms, fp64_peak, fp32_peak,
                                                       d["fp64_attempts"])},
        }

    # the plain FP64 tracer at the mixed tracer's tolerance: the equal-tolerance comparison
    fp64_at_mixed = None
    if "fp64" in res and "mixed" in res:
        c8 = headline_camera(relsim, relsim.PRECISION_FP64, args.side)
        c8.rtol, c8.atol = res["mixed"]["cam"].rtol, res["mixed"]["cam"].atol
        apply_tuned(tr, "fp64")
        d8 = time_device(tr, relsim, c8, n, ro, pix, flush, args.steps, args.warmup)
        ms8 = max_over_ranks(float(sum(d8["ms"])), ws, f"cuda:{local}")
        fp64_at_mixed = {"value": replica_value(n, ws, args.steps, ms8), "rtol": c8.rtol,
                         "attempts_per_ray": d8["attempts"] / (n * args.steps),
                         "ms_per_step": ms8 / args.steps}

    # stated error of the mixed tracer: every ray against the FP64 tracer's image
    if rank == 0 and "mixed" in res and not args.no_error_check:
        tr.set_launch_config()
        ref = tr.dispatch(headline_camera(relsim, relsim.PRECISION_FP64, args.side), fields=["status", "r_hit", "g"],
                          pixels=False)
        apply_tuned(tr, "mixed")
        out = tr.dispatch(res["mixed"]["cam"], fields=["status", "r_hit", "g"], pixels=False)
        summary["mixed"]["error_vs_fp64"] = error_vs_fp64(out, ref)

    serving = None
    if ws == 1 and not args.no_serving:
        import serve_stream

        torch.cuda.empty_cache()  # the server allocates its 120 GB budget arena up front
        s = serve_stream.run(check_requests=args.serving_check, device=local)
        err = s.get("error_vs_fp64") or {}
        serving = {"workload": s["workload"] + "; 10 % multi-source scenes of 2-16 holes (FP64)",
                   "served": s["served"], "failed": s["failed"], "multi_source": s["multi_source"],
                   "mrays_per_s": s["mrays_per_s"], "latency_ms_p50": s["latency_ms_p50"],
                   "latency_ms_p99": s["latency_ms_p99"], "latency_ms_max": s["latency_ms_max"],
                   "single_source_latency_ms_p50": s["single_source_latency_ms_p50"],
                   "single_source_latency_ms_p99": s["single_source_latency_ms_p99"],
                   "multi_source_latency_ms_p50": s["multi_source_latency_ms_p50"],
                   "multi_source_latency_ms_p99": s["multi_source_latency_ms_p99"],
                   "budget_bytes": s["budget_bytes"], "epochs": s["epochs"],
                   "error_vs_fp64": {k: v for k, v in err.items() if k != "per_request"} or None}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_port_baseline(relsim.camera_dict(res[headline]["cam"]), seconds=args.cpu_seconds)

    if rank == 0:
        h = summary[headline]
        two_pass = headline == "mixed" and not h["launch"].get("mixed_single_kernel", 0)
        launches_per_step = MIXED_TWO_PASS_LAUNCHES if two_pass else 1
        line = {
            "metric": METRIC, "value": h["value"], "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": h["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if headline == "fp64" else "f32+f64",
            "data": "synthetic camera grid",
            "config": {"workload": f"Kerr a=0.94 {args.side}^2 pinhole r=100 M i=17 deg FOV 12 deg, disk "
                                   f"[r_isco, 20 M], DP45; {headline} tracer at rtol=atol={h['rtol']:g}",
                       "precision": headline, "parallelism": f"replicas x{ws}",
                       "l2": "flushed between steps (256 MiB write)", "launch": h["launch"]},
            "msteps_per_s": h["msteps_per_s"],
            "attempts_per_ray": h["attempts_per_ray"],
            "latency_ms": {"kernel_p50": h["p50_ms"], "kernel_p99": h["p99_ms"],
                           "e2e_p50": 1e3 * float(np.percentile(lat, 50)),
                           "e2e_p99": 1e3 * float(np.percentile(lat, 99))},
            "roofline": h["roofline"],
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": H2D_BYTES_PER_IMAGE + SHADE_H2D_BYTES,
                    "d2h_bytes_per_step": d2h, "pixels": PIXELS_NOTE,
                    "call": "rt_dispatch into the 32-byte pixels, as dispatch_and_readback returns them",
                    "latency_ms_p50": 1e3 * float(np.percentile(lat, 50)),
                    "latency_ms_p99": 1e3 * float(np.percentile(lat, 99)),
                    "with_records": e2e_records},
            "gpu_launches": args.steps * launches_per_step,
            "gpu_launches_per_step": launches_per_step,
            "clocks": clocks,
            "fma_peak_tflops": {"fp64": fp64_peak, "fp32": fp32_peak},
            "precisions": summary,
        }
        if batched is not None:
            line["batched_c4"] = batched
        if bl is not None:
            line["boyer_lindquist"] = bl
        if serving is not None:
            line["serving"] = serving
        if cpu is not None:
            line["cpu_baseline"] = cpu
        # the precision comparison last, so that a cut tail of the line keeps it
        if "fp64" in summary:
            line["fp64_value"] = summary["fp64"]["value"]
        if fp64_at_mixed is not None:
            line["fp64_at_mixed_rtol"] = fp64_at_mixed
        if "fp64" in summary and "mixed" in summary:
            line["mixed_vs_fp64"] = summary["mixed"]["value"] / summary["fp64"]["value"]
            if fp64_at_mixed is not None:
                line["mixed_vs_fp64_at_mixed_rtol"] = summary["mixed"]["value"] / fp64_at_mixed["value"]
        print(json.dumps(line), flush=True)
    tr.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def vars_of(c) -> dict:
    return {f: getattr(c, f) for f, _ in c._fields_}


def executed_roofline(key, attempts, ms, fp64_peak, fp32_peak, fp64_attempts=None):
    """Executed floating-point work against the pipe peaks: per-attempt FP32 and
    FP64 FLOP counts from the committed ncu instruction mix of the same kernels
    (profiles/instruction_mix.json: FFMA and packed FFMA2 count 2 and 4 FLOP,
    FMUL/FADD 1 and 2, DFMA 2, DMUL/DADD 1), times the attempts of this run,
    over its device time.  The mixed tracer's attempts are weighted by pass:
    its FP32 attempts at the far pass's mix, its FP64 attempts (critical and
    near passes) at the near pass's.  None when no mix is committed for `key`."""
    path = os.path.join(ROOT, "profiles", "instruction_mix.json")
    try:
        with open(path) as f:
            mix = json.load(f)[key]
    except (OSError, ValueError, KeyError):
        return None
    sec = ms * 1e-3
    if "passes" in mix and fp64_attempts is not None:
        far, near = mix["passes"]["far"], mix["passes"]["near"]
        n32 = attempts - fp64_attempts
        f32_flop = n32 * far["fp32_flop_per_attempt"] + fp64_attempts * near["fp32_flop_per_attempt"]
        f64_flop = n32 * far["fp64_flop_per_attempt"] + fp64_attempts * near["fp64_flop_per_attempt"]
    else:
        f32_flop = attempts * mix["fp32_flop_per_attempt"]
        f64_flop = attempts * mix["fp64_flop_per_attempt"]
    f32 = f32_flop / sec / 1e12
    f64 = f64_flop / sec / 1e12
    return {"fp32_tflops": f32, "fp32_frac": f32 / fp32_peak, "fp64_tflops": f64, "fp64_frac": f64 / fp64_peak,
            "pipe_frac": f32 / fp32_peak + f64 / fp64_peak, "source": f"profiles/instruction_mix.json[{key}]"}


def committed_traffic(precision):
    """DRAM bytes per launch of the tracer kernel from the committed ncu summary, if present
    (precision 0: FP64, "bl": the Boyer-Lindquist kernel, else mixed)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(precision if isinstance(precision, str) else ("fp64" if precision == 0 else "mixed"))
    except (OSError, ValueError):
        return None


def error_vs_fp64(out: dict, ref: dict) -> dict:
    """Every ray of an image against the FP64 tracer's image of the same camera
    (the FP64 tracer is held to the FP64 oracle by the parity tests: classes
    exact outside the 1e-6 M band, radii and g to 1e-9)."""
    st, rst = out["status"], ref["status"]
    mism = int((st != rst).sum())
    both = (st == 3) & (rst == 3)
    rel = np.abs(out["r_hit"][both] - ref["r_hit"][both]) / ref["r_hit"][both]
    relg = np.abs(out["g"][both] - ref["g"][both]) / ref["g"][both]
    return {"rays": int(st.size), "class_mismatch_all_rays": mism, "disk_rays": int(both.sum()),
            "r_hit_rel_max": float(rel.max()) if rel.size else None,
            "r_hit_rel_p99": float(np.percentile(rel, 99)) if rel.size else None,
            "g_rel_max": float(relg.max()) if relg.size else None,
            "g_rel_p99": float(np.percentile(relg, 99)) if relg.size else None,
            "reference": "FP64 CUDA tracer, rtol 1e-10, same camera"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="both")
    ap.add_argument("--side", type=int, default=SIDE)
    ap.add_argument("--no-error-check", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-bundles", action="store_true", help="skip the 512-bundle batched measurement")
    ap.add_argument("--no-bl", action="store_true", help="skip the Boyer-Lindquist Kerr-Newman measurement")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream replay (one GPU only)")
    ap.add_argument("--serving-check", type=int, default=8,
                    help="single-source stream requests compared ray by ray with the FP64 tracer")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
