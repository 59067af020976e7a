"""Seeded synthetic scenes: the batched camera-bundle table and the request
stream (no dataset exists for this path; every scene is drawn here).

Bundle table (512 bundles, seed 0), one bundle per draw, in this order:
    side   = round32(exp U[ln 64, ln 1024])       (pixels, square image)
    a      = U[0, 0.998] M
    incl   = U[5, 85] deg
    r_obs  = exp U[ln 20, ln 500] M
    fov    = U[8, 40] deg
Disk [r_ISCO(a), 20 M]; M = 1; mixed precision unless asked otherwise.

Request stream (2000 requests, seed 1): Poisson arrivals at 200 requests/s;
each request draws its camera as a bundle above; 10 % of the requests are
multi-source Kerr-Schild superpositions of N ~ U{2..16} holes: the camera's
own hole at the origin (M = 1, spin a of the bundle) and N - 1 more, each with
mass U[0.2, 1] M, spin parameter U[0, 0.9] about an isotropic axis and
position U[-30, 30]^3 M.  A placement is drawn again when it lies within
2 (m_i + m_j) of another hole or within 5 + 2 m of the observer.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

import relsim


def round32(x: float) -> int:
    return max(32, int(round(x / 32.0)) * 32)


@dataclass
class BundleDraw:
    side: int
    spin: float
    incl_deg: float
    r_obs: float
    fov_deg: float

    def camera(self, precision: int = relsim.PRECISION_MIXED) -> relsim.Camera:
        return relsim.make_camera(spin=self.spin, r_obs=self.r_obs, incl_deg=self.incl_deg, fov_deg=self.fov_deg,
                                  width=self.side, height=self.side, precision=precision)


def _draw_bundle(rng: np.random.Generator) -> BundleDraw:
    side = round32(math.exp(rng.uniform(math.log(64.0), math.log(1024.0))))
    spin = rng.uniform(0.0, 0.998)
    incl = rng.uniform(5.0, 85.0)
    r_obs = math.exp(rng.uniform(math.log(20.0), math.log(500.0)))
    fov = rng.uniform(8.0, 40.0)
    return BundleDraw(side, spin, incl, r_obs, fov)


def bundle_table(n: int = 512, seed: int = 0) -> list[BundleDraw]:
    """The batched-bundle workload: n camera bundles of uneven size and geometry."""
    rng = np.random.default_rng(seed)
    return [_draw_bundle(rng) for _ in range(n)]


def bundle_cameras(n: int = 512, seed: int = 0, precision: int = relsim.PRECISION_MIXED) -> list[relsim.Camera]:
    return [d.camera(precision) for d in bundle_table(n, seed)]


@dataclass
class Source:
    mass: float
    spin_parameter: float  # a / m
    axis: tuple[float, float, float]
    position: tuple[float, float, float]


def rt_sources(sources: list[Source]) -> list[relsim.Source]:
    """The tracer's source records (each hole carries a disk [r_ISCO, 20 m])."""
    return [relsim.make_source(s.position, s.mass, s.spin_parameter, s.axis) for s in sources]


@dataclass
class Request:
    index: int
    arrival_s: float
    bundle: BundleDraw
    sources: list[Source] = field(default_factory=list)  # empty: the single Kerr hole of the bundle

    @property
    def multi_source(self) -> bool:
        return len(self.sources) > 0

    @property
    def rays(self) -> int:
        return self.bundle.side * self.bundle.side


def _isotropic_axis(rng: np.random.Generator) -> tuple[float, float, float]:
    z = rng.uniform(-1.0, 1.0)
    ph = rng.uniform(0.0, 2.0 * math.pi)
    s = math.sqrt(max(0.0, 1.0 - z * z))
    return (s * math.cos(ph), s * math.sin(ph), z)


def _draw_sources(rng: np.random.Generator, b: BundleDraw) -> list[Source]:
    """The N - 1 holes beside the camera's own (N ~ U{2..16} in total)."""
    n = int(rng.integers(2, 17)) - 1
    th = math.radians(b.incl_deg)
    observer = (b.r_obs * math.sin(th), 0.0, b.r_obs * math.cos(th))
    placed = [((0.0, 0.0, 0.0), 1.0)]  # the camera's hole
    out: list[Source] = []
    while len(out) < n:
        m = rng.uniform(0.2, 1.0)
        chi = rng.uniform(0.0, 0.9)
        axis = _isotropic_axis(rng)
        pos = tuple(float(v) for v in rng.uniform(-30.0, 30.0, 3))
        ok = math.dist(pos, observer) > 5.0 + 2.0 * m
        for q, mq in placed:
            ok = ok and math.dist(pos, q) > 2.0 * (m + mq)
        if ok:
            out.append(Source(m, chi, axis, pos))
            placed.append((pos, m))
    return out


def request_stream(n: int = 2000, rate_hz: float = 200.0, seed: int = 1, multi_fraction: float = 0.1
                   ) -> list[Request]:
    """The serving workload: Poisson arrivals, cameras as the bundle table, a
    fraction of multi-source scenes.  Draw order per request: inter-arrival
    gap, bundle, multi-source coin, sources."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate_hz)
        b = _draw_bundle(rng)
        multi = rng.uniform() < multi_fraction
        srcs = _draw_sources(rng, b) if multi else []
        out.append(Request(i, t, b, srcs))
    return out
