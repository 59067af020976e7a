"""Autotuner of the persistent tracer's launch shape.

Sweeps block size, persistent CTAs per SM and the warp refill threshold on a
representative camera, times each with CUDA events (best of `reps` after a
warm-up, outputs resident on the device) and writes the fastest configuration
per precision to tuned_launch.json beside this file.  Tracer users apply it
with `apply_tuned(tracer, precision)`.

    python relativity-simulator_b200/autotune.py [--side 1024] [--precision fp64|mixed|both]
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import relsim  # noqa: E402

TUNED = os.path.join(HERE, "tuned_launch.json")
BLOCKS = (64, 128, 256)
THRESHOLDS = (1, 2, 4, 8, 16, 32)
RAYS_PER_THREAD = (1, 4)
ROLLED = (0, 1)


def load_tuned() -> dict:
    try:
        with open(TUNED) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def apply_tuned(tracer: relsim.Tracer, precision: str) -> dict | None:
    cfg = load_tuned().get(precision)
    if cfg:
        tracer.set_launch_config(cfg["block_size"], cfg["ctas_per_sm"], cfg["refill_threshold"],
                                 cfg.get("rays_per_thread", 0), cfg.get("fp64_rolled", 0))
    return cfg


def time_config(tr, cam, ro, pix_ptr, n, block, ctas, thr, rpt, rolled, reps=3) -> float:
    tr.set_launch_config(block, ctas, thr, rpt, rolled)
    tr.dispatch_device(cam, ro, pix_ptr, n)
    tr.stats()
    best = float("inf")
    for _ in range(reps):
        tr.dispatch_device(cam, ro, pix_ptr, n)
        best = min(best, tr.stats().kernel_ms)
    return best


def tune(tr: relsim.Tracer, precision: str, side: int = 1024, verbose: bool = True) -> dict:
    import torch

    prec = relsim.PRECISION_MIXED if precision == "mixed" else relsim.PRECISION_FP64
    cam = relsim.make_camera(spin=0.94, r_obs=100.0, incl_deg=17.0, fov_deg=12.0, width=side, height=side,
                             precision=prec)
    n = side * side
    ro, _t = relsim.device_ray_out(n, ["status", "r", "theta", "phi", "r_hit", "g"])
    pix = torch.empty(n * 32, dtype=torch.uint8, device="cuda")
    results = []
    rolled_opts = ROLLED if precision == "fp64" else (1,)
    seen = set()
    for block, thr, rpt, rolled in itertools.product(BLOCKS, THRESHOLDS, RAYS_PER_THREAD, rolled_opts):
        tr.set_launch_config(block, 0, thr, rpt, rolled)
        eff = tr.launch_config()
        occ = eff.ctas_per_sm
        for ctas in sorted({occ, max(1, occ - 1)}):
            key = (eff.block_size, ctas, thr, rpt, rolled)
            if key in seen:
                continue
            seen.add(key)
            ms = time_config(tr, cam, ro, pix.data_ptr(), n, eff.block_size, ctas, thr, rpt, rolled)
            results.append({"block_size": eff.block_size, "ctas_per_sm": ctas, "refill_threshold": thr,
                            "rays_per_thread": rpt, "fp64_rolled": rolled, "ms": ms, "mrays_per_s": n / ms / 1e3})
            if verbose:
                print(json.dumps(results[-1]), flush=True)
    best = min(results, key=lambda r: r["ms"])
    tr.set_launch_config(0, 0, 0, 0, 0)
    return {"best": best, "sweep": results, "camera": f"Kerr a=0.94 {side}^2 r=100 i=17 FOV 12"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--side", type=int, default=1024)
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="fp64")
    a = ap.parse_args()
    tuned = load_tuned()
    with relsim.Tracer(0) as tr:
        for prec in (["fp64", "mixed"] if a.precision == "both" else [a.precision]):
            res = tune(tr, prec, a.side)
            b = res["best"]
            tuned[prec] = {k: b[k] for k in ("block_size", "ctas_per_sm", "refill_threshold", "rays_per_thread",
                                             "fp64_rolled")}
            tuned[prec]["mrays_per_s_at_tuning"] = b["mrays_per_s"]
            tuned[prec]["tuned_on"] = res["camera"]
    with open(TUNED, "w") as f:
        json.dump(tuned, f, indent=1)
    print(json.dumps(tuned))


if __name__ == "__main__":
    main()
