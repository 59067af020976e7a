"""Trace one image on cuda:0 and print a summary (also the profiling driver).

    python relativity-simulator_b200/trace_once.py [--side 512] [--spin 0.94] [--r-obs 100]
        [--incl 17] [--fov 12] [--precision fp64|mixed] [--repeat 1]
        [--metric ks|bl] [--charge 0] [--sources N] [--device] [--shade]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np  # noqa: E402

import relsim  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--side", type=int, default=512)
    ap.add_argument("--spin", type=float, default=0.94)
    ap.add_argument("--r-obs", type=float, default=100.0)
    ap.add_argument("--incl", type=float, default=17.0)
    ap.add_argument("--fov", type=float, default=12.0)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--refill", type=int, default=0)
    ap.add_argument("--rays-per-thread", type=int, default=0)
    ap.add_argument("--fp64-rolled", type=int, default=0)
    ap.add_argument("--rtol", type=float, default=None)
    ap.add_argument("--fp64-radius", type=float, default=0.0)
    ap.add_argument("--critical-band", type=float, default=0.0,
                    help="mixed precision: near-critical band in M traced in FP64 (0: 1 M, negative: none)")
    ap.add_argument("--mixed-single", type=int, default=0,
                    help="mixed precision: 1 = the single-kernel form instead of far/near passes")
    ap.add_argument("--metric", choices=["ks", "bl"], default="ks",
                    help="ks: Kerr-Schild Hamiltonian tracer; bl: Boyer-Lindquist Kerr-Newman tracer (FP64)")
    ap.add_argument("--charge", type=float, default=0.0, help="Kerr-Newman charge Q (--metric bl)")
    ap.add_argument("--sources", type=int, default=0,
                    help="multi-source scene: the first request of the seeded stream with this many bodies beside "
                         "the camera's hole (its camera at --side and --precision), traced by the multi-source tracer")
    ap.add_argument("--device", action="store_true",
                    help="device-resident outputs (rt_dispatch_device: one set of launches, no host bands)")
    ap.add_argument("--shade", action="store_true",
                    help="shade the pixels (rt_set_shading defaults): rays are followed through the translucent disk")
    ap.add_argument("--sky", action="store_true",
                    help="shade with the procedural sky on (the default sky profile; implies --shade)")
    ap.add_argument("--record", choices=["minimal", "bench"], default="minimal",
                    help="outputs written: class and step counts, or the bench's record (class, r, theta, "
                         "phi, r_hit, g) plus the 32-byte pixels")
    a = ap.parse_args()
    cam = relsim.make_camera(spin=a.spin, r_obs=a.r_obs, incl_deg=a.incl, fov_deg=a.fov, width=a.side,
                             height=a.side,
                             precision=relsim.PRECISION_MIXED if a.precision == "mixed" else relsim.PRECISION_FP64,
                             rtol=a.rtol, mixed_fp64_radius=a.fp64_radius, critical_band=a.critical_band,
                             metric_form=relsim.METRIC_BOYER_LINDQUIST if a.metric == "bl" else relsim.METRIC_KERR_SCHILD,
                             charge=a.charge)
    srcs = None
    if a.sources > 0:
        import scenes

        req = [r for r in scenes.request_stream() if r.multi_source and len(r.sources) == a.sources][0]
        cam = req.bundle.camera(relsim.PRECISION_MIXED if a.precision == "mixed" else relsim.PRECISION_FP64)
        cam.screen_width = cam.screen_height = a.side
        if a.rtol is not None:
            cam.rtol = cam.atol = a.rtol
        srcs = scenes.rt_sources(req.sources)
    with relsim.Tracer(0) as tr:
        tr.set_launch_config(a.block, 0, a.refill, a.rays_per_thread, a.fp64_rolled, a.mixed_single)
        if a.shade or a.sky:
            tr.set_shading(relsim.shading(sky_enabled=1) if a.sky else relsim.shading())
        dev = None
        if a.device:
            import torch

            n = cam.screen_width * cam.screen_height
            fields = ["status", "r", "theta", "phi", "r_hit", "g"] if a.record == "bench" else ["status"]
            dev = relsim.device_ray_out(n, fields) + (torch.empty(n * 32, dtype=torch.uint8, device="cuda"),)
        for _ in range(a.repeat):
            if dev is not None:
                tr.dispatch_device(cam, dev[0], dev[2].data_ptr(), cam.screen_width * cam.screen_height)
                tr.synchronize()
                out = {"status": dev[1]["status"].cpu().numpy().view(np.uint32)}
            elif srcs is not None:
                out = tr.dispatch_multi(cam, srcs, fields=["status", "steps_accepted", "steps_rejected"],
                                        pixels=False)
            elif a.record == "bench":
                out = tr.dispatch(cam, fields=["status", "r", "theta", "phi", "r_hit", "g"], pixels=True)
            else:
                out = tr.dispatch(cam, fields=["status", "steps_accepted", "steps_rejected"], pixels=False)
            s = tr.stats()
    print(json.dumps({"rays": int(s.rays), "attempts": int(s.attempts), "accepted": int(s.accepted),
                      "fp64_attempts": int(s.fp64_attempts), "rhs_evals": int(s.rhs_evals),
                      "kernel_ms": s.kernel_ms, "mrays_per_s": s.rays / s.kernel_ms / 1e3 if s.kernel_ms > 0 else None,
                      "classes": np.bincount(out["status"], minlength=4).tolist(),
                      **attempt_tail(out)}))


def attempt_tail(out: dict) -> dict:
    """Largest and 99.9th-percentile step attempts of one ray (host records with step counts)."""
    if "steps_accepted" not in out:
        return {}
    att = out["steps_accepted"].astype(np.int64) + out["steps_rejected"]
    return {"ray_attempts_max": int(att.max()), "ray_attempts_p999": float(np.percentile(att, 99.9)),
            "ray_attempts_mean": float(att.mean())}


if __name__ == "__main__":
    main()
