"""Camera configurations of the benchmark cases, shared by tests and fixtures.

c1  Schwarzschild a=0, 256^2, observer r=50 M, inclination 60 deg, FOV 30 deg,
    disk [6, 20] M
c2  Kerr a=0.94, 2048^2, r=100 M, 17 deg, FOV 12 deg, disk [r_ISCO, 20] M
c3  Kerr a=0.998, 4096^2, r=60 M, 80 deg, FOV 20 deg, disk [r_ISCO, 20] M
All: DP45 rtol = atol = 1e-10, <= 20000 attempts, captured r < 1.01 r_+,
escaped r > 1000 M.
"""
from __future__ import annotations

import relsim

CONFIGS = {
    "c1": dict(spin=0.0, r_obs=50.0, incl_deg=60.0, fov_deg=30.0, width=256, height=256, disk_inner=6.0),
    "c2": dict(spin=0.94, r_obs=100.0, incl_deg=17.0, fov_deg=12.0, width=2048, height=2048),
    "c3": dict(spin=0.998, r_obs=60.0, incl_deg=80.0, fov_deg=20.0, width=4096, height=4096),
}


def config_cam(tag: str, **over) -> relsim.Camera:
    kw = dict(CONFIGS[tag])
    kw.update(over)
    return relsim.make_camera(**kw)


def config_camera(tag: str, **over) -> dict:
    """The configuration as the oracle's camera dict."""
    return relsim.camera_dict(config_cam(tag, **over))
