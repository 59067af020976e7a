"""Python binding of the tracer's C ABI (include/relsim_cuda.h).

The product is the CUDA library librelsim_cuda.so; this module loads it with
ctypes and exposes the same entry points to Python callers (tests, bench,
serving loop).  There is no CPU path: if the library or the GPU is missing,
`Tracer()` raises.

    from relsim import Tracer, make_camera
    tr = Tracer()
    cam = make_camera(spin=0.94, r_obs=100, incl_deg=17, fov_deg=12, width=2048, height=2048)
    out = tr.dispatch(cam)            # host arrays: status, r, theta, phi, r_hit, g, ...
"""
from __future__ import annotations

import ctypes
import math
import os
from typing import Iterable

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RELSIM_LIB") or os.path.join(HERE, "librelsim_cuda.so")

RT_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "TIMEOUT", 4: "DEVICE", 5: "CANCELLED", 6: "NOT_READY",
                7: "BUDGET", 8: "AGAIN"}
RAY_UNFINISHED, RAY_CAPTURED, RAY_ESCAPED, RAY_DISK = 0, 1, 2, 3
RAYFLAG_NONFINITE, RAYFLAG_STEP_UNDERFLOW, RAYFLAG_MAX_STEPS, RAYFLAG_EARLY_CAPTURE = 1, 2, 4, 8
PIXEL_HORIZON_ABSORBED, PIXEL_CELESTIAL_HIT, PIXEL_ACCRETION_DISK_HIT = 1, 2, 4
PRECISION_FP64, PRECISION_MIXED = 0, 1
METRIC_KERR_SCHILD, METRIC_BOYER_LINDQUIST = 0, 1  # rt_metric_form
MIXED_RTOL = 1e-8  # DP45 tolerance of the mixed-precision mode

_d = ctypes.c_double
_u32 = ctypes.c_uint32


class Camera(ctypes.Structure):
    _fields_ = [
        ("observer_position", _d * 4), ("tetrad_e1", _d * 4), ("tetrad_e2", _d * 4), ("tetrad_e3", _d * 4),
        ("field_of_view_rad", _d), ("metric_mass", _d), ("metric_spin", _d), ("escape_radius", _d),
        ("capture_scale", _d), ("disk_inner_radius", _d), ("disk_outer_radius", _d), ("rtol", _d), ("atol", _d),
        ("step_cap_fraction", _d), ("initial_step_fraction", _d), ("projection_tol", _d), ("mixed_fp64_radius", _d),
        ("metric_charge", _d), ("mixed_critical_band", _d),
        ("screen_width", _u32), ("screen_height", _u32), ("max_integration_steps", _u32), ("early_capture", _u32),
        ("precision_mode", _u32), ("dispatch_row_offset", _u32), ("dispatch_row_count", _u32),
        ("tile_origin_x", _u32), ("tile_origin_y", _u32), ("tile_extent_x", _u32), ("tile_extent_y", _u32),
        ("metric_form", _u32),
    ]


class DiskProfile(ctypes.Structure):
    """rt_disk_profile: GpuDiskProfile's 32 floats in the reference's order."""
    _fields_ = [(n, ctypes.c_float) for n in (
        "enabled", "inner_radius_scale", "outer_radius_mass_units", "peak_temperature_k", "floor_temperature_k",
        "temperature_exponent", "zero_torque_strength", "extra_beaming_exponent", "brightness", "color_saturation",
        "tint_strength", "opacity_scale", "tint_r", "tint_g", "tint_b", "rotation_speed_scale", "ring_amplitude",
        "ring_frequency", "ring_sharpness", "spiral_arm_count", "spiral_pitch", "spiral_amplitude",
        "turbulence_amplitude", "turbulence_scale", "turbulence_octaves", "radial_stretch", "grain_amplitude",
        "grain_scale", "reference_luminance", "noise_seed", "temperature_normalization", "edge_softness")]


class SkyProfile(ctypes.Structure):
    """rt_sky_profile: the GpuSkyProfile image (1808 bytes); fields by name through
    sky_profile() / sky_get()."""
    _fields_ = [("bytes", ctypes.c_uint8 * 1808)]


class Shading(ctypes.Structure):
    """rt_shading: the pixel shading tail (disk colour, the procedural sky, tonemapping)."""
    _fields_ = [("disk", DiskProfile), ("disk_temperature_scale_k", _d), ("disk_temperature_floor_k", _d),
                ("disk_color_saturation", _d), ("disk_doppler_beaming_exponent", _d), ("time", _d),
                ("camera_exposure", _d), ("tonemapping_mode", _u32), ("hydro_model", _u32),
                ("accretion_rate_scale", ctypes.c_float), ("sky_enabled", _u32), ("sky", SkyProfile),
                ("torus_inner_radius", ctypes.c_float), ("torus_center_radius", ctypes.c_float),
                ("adiabatic_index", ctypes.c_float), ("optical_depth_scale", ctypes.c_float),
                ("sampling_density", ctypes.c_float), ("reserved_torus", ctypes.c_float)]


class PixelOut(ctypes.Structure):
    _fields_ = [("r", ctypes.c_float), ("g", ctypes.c_float), ("b", ctypes.c_float), ("a", ctypes.c_float),
                ("redshift", ctypes.c_float), ("affine_parameter", ctypes.c_float), ("status_flags", _u32),
                ("iterations_used", _u32)]


RAY_FIELDS = [("status", np.uint32), ("flags", np.uint32), ("steps_accepted", np.uint32),
              ("steps_rejected", np.uint32), ("r", np.float64), ("theta", np.float64), ("phi", np.float64),
              ("r_hit", np.float64), ("g", np.float64), ("lambda", np.float64), ("dH", np.float64),
              ("dE", np.float64), ("dLz", np.float64), ("dQ", np.float64), ("exit_x", np.float64),
              ("exit_y", np.float64), ("exit_z", np.float64), ("body", np.uint32)]
BODY_NONE = 0xFFFFFFFF  # RT_BODY_NONE
PIXEL_DTYPE = np.dtype([("r", "f4"), ("g", "f4"), ("b", "f4"), ("a", "f4"), ("redshift", "f4"),
                        ("affine_parameter", "f4"), ("status_flags", "u4"), ("iterations_used", "u4")])


class RayOut(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name, _ in RAY_FIELDS]


class LaunchConfig(ctypes.Structure):
    _fields_ = [("block_size", _u32), ("ctas_per_sm", _u32), ("refill_threshold", _u32), ("rays_per_thread", _u32),
                ("fp64_rolled", _u32), ("mixed_single_kernel", _u32)]


class Stats(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_uint64), ("attempts", ctypes.c_uint64), ("accepted", ctypes.c_uint64),
                ("rhs_evals", ctypes.c_uint64), ("fp64_attempts", ctypes.c_uint64), ("kernel_ms", _d)]


class Source(ctypes.Structure):
    """rt_source: a black-hole body beside the camera's hole (multi-source scenes)."""
    _fields_ = [("position", _d * 3), ("mass", _d), ("spin_parameter", _d), ("axis", _d * 3), ("disk_enabled", _d),
                ("disk_inner_scale", _d), ("disk_outer_units", _d), ("disk", DiskProfile)]


MAX_SOURCES = 16  # RT_MAX_SOURCES: the camera's hole and up to 15 sources
RAYFLAG_DIVERGED = 16


def make_source(position, mass: float = 1.0, spin_parameter: float = 0.0, axis=(0.0, 0.0, 1.0), disk: bool = True,
                disk_inner_scale: float = 1.0, disk_outer_units: float = 20.0,
                profile: "DiskProfile | None" = None) -> Source:
    """A body; its disk appearance defaults to GpuDiskProfile's defaults (rt_shading_defaults' disk)."""
    if profile is None:
        profile = shading().disk
    return Source((_d * 3)(*position), mass, spin_parameter, (_d * 3)(*axis), 1.0 if disk else 0.0, disk_inner_scale,
                  disk_outer_units, profile)


class ServerConfig(ctypes.Structure):
    _fields_ = [("memory_budget_bytes", ctypes.c_uint64), ("max_requests", _u32), ("chunk_rays", _u32),
                ("epoch_rays", _u32), ("max_epoch_bundles", _u32), ("record_mask", _u32), ("min_epoch_rays", _u32),
                ("launch_fp64", LaunchConfig), ("launch_mixed", LaunchConfig), ("multi_source_sms", _u32),
                ("reserved", _u32)]


class RequestDone(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("rays", ctypes.c_uint64), ("latency_ms", _d), ("queue_ms", _d),
                ("status", ctypes.c_int), ("reserved", _u32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("requests_submitted", ctypes.c_uint64), ("requests_done", ctypes.c_uint64),
                ("rays_done", ctypes.c_uint64), ("epochs", ctypes.c_uint64), ("bundles", ctypes.c_uint64),
                ("bytes_in_use", ctypes.c_uint64), ("peak_bytes_in_use", ctypes.c_uint64),
                ("budget_bytes", ctypes.c_uint64), ("pending", _u32), ("peak_active", _u32),
                ("peak_epoch_rays", ctypes.c_uint64)]


# record_mask bits: rt_ray_out fields in declaration order, then the pixels
RECORD_BIT = {name: 1 << i for i, (name, _) in enumerate(
    [("status", 0), ("flags", 0), ("steps_accepted", 0), ("steps_rejected", 0), ("r", 0), ("theta", 0),
     ("phi", 0), ("r_hit", 0), ("g", 0), ("lambda", 0), ("dH", 0), ("dE", 0), ("dLz", 0), ("dQ", 0)])}
RECORD_BIT["pixels"] = 1 << 14

_lib: ctypes.CDLL | None = None

EXPORTS = ["rt_create", "rt_destroy", "rt_is_ready", "rt_is_platform_supported", "rt_last_error", "rt_abi_version",
           "rt_camera_defaults", "rt_camera_look_at_hole", "rt_dispatch", "rt_dispatch_tile", "rt_dispatch_device",
           "rt_trace_bundles_device", "rt_bundle_rays", "rt_set_launch_config", "rt_get_launch_config",
           "rt_get_stats", "rt_synchronize", "rt_measure_fma_peak", "rt_trace_bundles_noalloc", "rt_kerr_isco_radius", "rt_dispatch_multi", "rt_dispatch_multi_device",
           "rt_server_config_defaults", "rt_server_create", "rt_server_destroy", "rt_server_submit",
           "rt_server_poll", "rt_server_get_stats", "rt_server_last_error", "rt_server_submit_multi",
           "rt_shading_defaults", "rt_set_shading", "rt_server_set_shading", "rt_sky_profile_defaults",
           "rt_sky_profile_set", "rt_sky_profile_get"]
NOALLOC_MAX_BUNDLES = 32  # RT_NOALLOC_MAX_BUNDLES


def lib() -> ctypes.CDLL:
    """Load librelsim_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: run relativity-simulator_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        v, p = ctypes.c_void_p, ctypes.POINTER
        L.rt_create.argtypes = [p(ctypes.c_void_p), ctypes.c_int]
        L.rt_destroy.argtypes = [v]
        L.rt_destroy.restype = None
        L.rt_is_ready.argtypes = [v]
        L.rt_last_error.argtypes = [v]
        L.rt_last_error.restype = ctypes.c_char_p
        L.rt_camera_defaults.argtypes = [p(Camera)]
        L.rt_camera_defaults.restype = None
        L.rt_camera_look_at_hole.argtypes = [p(Camera), _d, _d, _d]
        L.rt_camera_look_at_hole.restype = None
        L.rt_dispatch.argtypes = [v, p(Camera), v, p(RayOut), ctypes.c_size_t, v]
        L.rt_dispatch_tile.argtypes = [v, p(Camera), v, p(RayOut), ctypes.c_size_t]
        L.rt_dispatch_device.argtypes = [v, p(Camera), v, p(RayOut), ctypes.c_size_t, v]
        L.rt_trace_bundles_device.argtypes = [v, p(Camera), _u32, v, v, p(RayOut), ctypes.c_size_t, v]
        L.rt_bundle_rays.argtypes = [p(Camera), _u32]
        L.rt_bundle_rays.restype = ctypes.c_uint64
        L.rt_set_launch_config.argtypes = [v, p(LaunchConfig)]
        L.rt_shading_defaults.argtypes = [p(Shading)]
        L.rt_shading_defaults.restype = None
        L.rt_sky_profile_defaults.argtypes = [p(SkyProfile)]
        L.rt_sky_profile_defaults.restype = None
        L.rt_sky_profile_set.argtypes = [p(SkyProfile), ctypes.c_char_p, _d]
        L.rt_sky_profile_set.restype = ctypes.c_int
        L.rt_sky_profile_get.argtypes = [p(SkyProfile), ctypes.c_char_p, p(_d)]
        L.rt_sky_profile_get.restype = ctypes.c_int
        L.rt_set_shading.argtypes = [v, p(Shading)]
        L.rt_server_set_shading.argtypes = [v, p(Shading)]
        L.rt_get_launch_config.argtypes = [v, p(LaunchConfig)]
        L.rt_get_stats.argtypes = [v, p(Stats)]
        L.rt_synchronize.argtypes = [v, _d]
        L.rt_measure_fma_peak.argtypes = [v, p(_d), p(_d)]
        L.rt_dispatch_multi.argtypes = [v, p(Camera), p(Source), _u32, v, p(RayOut), ctypes.c_size_t]
        L.rt_dispatch_multi_device.argtypes = [v, p(Camera), p(Source), _u32, v, p(RayOut), ctypes.c_size_t, v]
        L.rt_kerr_isco_radius.argtypes = [_d, _d]
        L.rt_kerr_isco_radius.restype = _d
        L.rt_server_config_defaults.argtypes = [p(ServerConfig)]
        L.rt_server_config_defaults.restype = None
        L.rt_server_create.argtypes = [p(ctypes.c_void_p), ctypes.c_int, p(ServerConfig)]
        L.rt_server_destroy.argtypes = [v]
        L.rt_server_destroy.restype = None
        L.rt_server_submit.argtypes = [v, p(Camera), v, p(RayOut), ctypes.c_size_t, p(ctypes.c_uint64)]
        L.rt_server_submit_multi.argtypes = [v, p(Camera), p(Source), _u32, v, p(RayOut), ctypes.c_size_t,
                                             p(ctypes.c_uint64)]
        L.rt_server_poll.argtypes = [v, p(RequestDone), _u32, p(_u32), _d]
        L.rt_server_get_stats.argtypes = [v, p(ServerStats)]
        L.rt_server_last_error.argtypes = [v]
        L.rt_server_last_error.restype = ctypes.c_char_p
        L.rt_trace_bundles_noalloc.argtypes = [ctypes.c_int, p(Camera), _u32, v, v, p(RayOut), ctypes.c_size_t,
                                               p(LaunchConfig), v, ctypes.c_char_p, ctypes.c_size_t]
        _lib = L
    return _lib


class RelsimError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def make_camera(*, spin: float = 0.94, mass: float = 1.0, r_obs: float = 100.0, incl_deg: float = 17.0,
                phi_obs: float = 0.0, fov_deg: float = 12.0, width: int = 2048, height: int = 2048,
                escape_radius: float = 1000.0, capture_scale: float = 1.01, disk_inner: float = 0.0,
                disk_outer: float = 20.0, rtol: float | None = None, atol: float | None = None,
                max_steps: int = 20000,
                step_cap: float = 0.1, h0: float = 0.01, projection_tol: float = 1e-12, early_capture: bool = True,
                precision: int = PRECISION_FP64, mixed_fp64_radius: float = 0.0, row_offset: int = 0,
                row_count: int = 0, metric_form: int = METRIC_KERR_SCHILD, charge: float = 0.0,
                critical_band: float = 0.0) -> Camera:
    """A camera looking at the hole from (r_obs, incl, phi_obs) with a static-observer tetrad.

    metric_form METRIC_BOYER_LINDQUIST traces the Kerr-Newman metric of the
    given charge in Boyer-Lindquist coordinates (FP64, ZAMO observer).

    critical_band (mixed mode): rays whose constants lie within this many M of
    the critical curve are traced in FP64 from their first step (0: 1 M,
    negative: none).

    Tolerances default to rtol = atol = 1e-10 for FP64 and 1e-8 for the mixed
    precision mode (whose FP32 stages carry ~1e-7 relative increments)."""
    if rtol is None:
        rtol = MIXED_RTOL if precision == PRECISION_MIXED else 1e-10
    if atol is None:
        atol = rtol
    c = Camera()
    c.field_of_view_rad = math.radians(fov_deg)
    c.metric_mass, c.metric_spin = mass, spin
    c.escape_radius, c.capture_scale = escape_radius, capture_scale
    c.disk_inner_radius, c.disk_outer_radius = disk_inner, disk_outer
    c.rtol, c.atol = rtol, atol
    c.step_cap_fraction, c.initial_step_fraction, c.projection_tol = step_cap, h0, projection_tol
    c.mixed_fp64_radius, c.mixed_critical_band = mixed_fp64_radius, critical_band
    c.screen_width, c.screen_height = width, height
    c.max_integration_steps = max_steps
    c.early_capture = 1 if early_capture else 0
    c.precision_mode = precision
    c.dispatch_row_offset, c.dispatch_row_count = row_offset, row_count
    c.metric_form, c.metric_charge = metric_form, charge
    th, ph = math.radians(incl_deg), phi_obs
    st, ct, sp, cp = math.sin(th), math.cos(th), math.sin(ph), math.cos(ph)
    er, eth, eph = (st * cp, st * sp, ct), (ct * cp, ct * sp, -st), (-sp, cp, 0.0)
    c.observer_position[:] = [0.0, r_obs, th, ph]
    c.tetrad_e1[:] = [0.0, -er[0], -er[1], -er[2]]
    c.tetrad_e2[:] = [0.0, *eph]
    c.tetrad_e3[:] = [0.0, -eth[0], -eth[1], -eth[2]]
    return c


def camera_dict(c: Camera) -> dict:
    """The camera as a dict of plain values (the oracle's camera keys)."""
    d = {}
    for name, _ in Camera._fields_:
        v = getattr(c, name)
        d[name] = list(v) if hasattr(v, "__len__") else v
    d["max_steps"] = c.max_integration_steps
    return d


def window_rays(c: Camera) -> int:
    rows = c.screen_height - min(c.dispatch_row_offset, c.screen_height)
    if c.dispatch_row_count:
        rows = min(rows, c.dispatch_row_count)
    return c.screen_width * rows


class Tracer:
    """One device handle (VulkanComputeExecutor's role)."""

    def __init__(self, device: int = 0):
        L = lib()
        h = ctypes.c_void_p()
        st = L.rt_create(ctypes.byref(h), device)
        if st != RT_OK:
            raise RelsimError(st, f"rt_create(device={device}) failed (no sm_100 device?)")
        self._h = h
        self.lib = L

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.rt_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def _check(self, st: int) -> None:
        if st != RT_OK:
            raise RelsimError(st, self.lib.rt_last_error(self._h).decode())

    def is_ready(self) -> bool:
        return bool(self.lib.rt_is_ready(self._h))

    def dispatch(self, cam: Camera, fields: Iterable[str] | None = None, pixels: bool = True,
                 cancel: ctypes.c_int | None = None, tile: bool = False) -> dict:
        """Trace on the device, read back into new host arrays (rt_dispatch / rt_dispatch_tile)."""
        names = [n for n, _ in RAY_FIELDS] if fields is None else list(fields)
        if tile:
            n = min(cam.tile_extent_x, cam.screen_width - cam.tile_origin_x) * \
                min(cam.tile_extent_y, cam.screen_height - cam.tile_origin_y)
        else:
            n = window_rays(cam)
        out = {}
        ro = RayOut()
        for name, dt in RAY_FIELDS:
            if name in names:
                out[name] = np.empty(n, dtype=dt)
                setattr(ro, name, out[name].ctypes.data)
        pix = np.empty(n, dtype=PIXEL_DTYPE) if pixels else None
        pptr = pix.ctypes.data if pix is not None else None
        if tile:
            st = self.lib.rt_dispatch_tile(self._h, ctypes.byref(cam), pptr, ctypes.byref(ro), n)
        else:
            st = self.lib.rt_dispatch(self._h, ctypes.byref(cam), pptr, ctypes.byref(ro), n,
                                      ctypes.byref(cancel) if cancel is not None else None)
        self._check(st)
        if pix is not None:
            out["pixels"] = pix
        return out

    def dispatch_multi(self, cam: Camera, sources: list[Source], fields: Iterable[str] | None = None,
                       pixels: bool = True) -> dict:
        """Trace a multi-source scene (the camera's hole plus `sources`) into new host arrays."""
        names = [n for n, _ in RAY_FIELDS] if fields is None else list(fields)
        n = window_rays(cam)
        out = {}
        ro = RayOut()
        for name, dt in RAY_FIELDS:
            if name in names:
                out[name] = np.empty(n, dtype=dt)
                setattr(ro, name, out[name].ctypes.data)
        pix = np.empty(n, dtype=PIXEL_DTYPE) if pixels else None
        arr = (Source * max(len(sources), 1))(*sources)
        self._check(self.lib.rt_dispatch_multi(self._h, ctypes.byref(cam), arr, len(sources),
                                               pix.ctypes.data if pix is not None else None, ctypes.byref(ro), n))
        if pix is not None:
            out["pixels"] = pix
        return out

    def dispatch_multi_device(self, cam: Camera, sources: list[Source], rays: RayOut, pixels_ptr: int | None,
                              capacity: int, stream: int | None = None) -> None:
        arr = (Source * max(len(sources), 1))(*sources)
        self._check(self.lib.rt_dispatch_multi_device(self._h, ctypes.byref(cam), arr, len(sources), pixels_ptr,
                                                      ctypes.byref(rays), capacity, stream))

    def dispatch_device(self, cam: Camera, rays: RayOut, pixels_ptr: int | None, capacity: int,
                        stream: int | None = None) -> None:
        """Enqueue a trace into device buffers (pointers from torch tensors); no wait."""
        self._check(self.lib.rt_dispatch_device(self._h, ctypes.byref(cam), pixels_ptr, ctypes.byref(rays),
                                                capacity, stream))

    def trace_bundles_device(self, cams: list[Camera], rays: RayOut, pixels_ptr: int | None, capacity: int,
                             offsets: np.ndarray | None = None, stream: int | None = None) -> None:
        arr = (Camera * len(cams))(*cams)
        optr = None
        if offsets is not None:
            offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
            optr = offsets.ctypes.data
        self._check(self.lib.rt_trace_bundles_device(self._h, arr, len(cams), optr, pixels_ptr, ctypes.byref(rays),
                                                     capacity, stream))

    def stats(self) -> Stats:
        s = Stats()
        self._check(self.lib.rt_get_stats(self._h, ctypes.byref(s)))
        return s

    def synchronize(self, timeout_ms: float = 0.0) -> None:
        self._check(self.lib.rt_synchronize(self._h, timeout_ms))

    def set_shading(self, shading: "Shading | None") -> None:
        """Shade the pixels of later dispatches (None: colour off)."""
        self._check(self.lib.rt_set_shading(self._h, ctypes.byref(shading) if shading is not None else None))

    def set_launch_config(self, block_size: int = 0, ctas_per_sm: int = 0, refill_threshold: int = 0,
                          rays_per_thread: int = 0, fp64_rolled: int = 0, mixed_single_kernel: int = 0) -> None:
        c = LaunchConfig(block_size, ctas_per_sm, refill_threshold, rays_per_thread, fp64_rolled, mixed_single_kernel)
        self._check(self.lib.rt_set_launch_config(self._h, ctypes.byref(c)))

    def launch_config(self) -> LaunchConfig:
        c = LaunchConfig()
        self._check(self.lib.rt_get_launch_config(self._h, ctypes.byref(c)))
        return c

    def measure_fma_peak(self) -> tuple[float, float]:
        f64, f32 = _d(), _d()
        self._check(self.lib.rt_measure_fma_peak(self._h, ctypes.byref(f64), ctypes.byref(f32)))
        return f64.value, f32.value


def trace_bundles_noalloc(cams: list[Camera], rays: RayOut, pixels_ptr: int | None, capacity: int,
                          offsets: np.ndarray | None = None, device: int = 0, launch: LaunchConfig | None = None,
                          stream: int | None = None) -> None:
    """rt_trace_bundles_noalloc: the bundle trace without a handle and without
    device allocation (scratch in a static device array); enqueued, no wait."""
    arr = (Camera * len(cams))(*cams)
    optr = None
    if offsets is not None:
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        optr = offsets.ctypes.data
    err = ctypes.create_string_buffer(256)
    st = lib().rt_trace_bundles_noalloc(device, arr, len(cams), optr, pixels_ptr, ctypes.byref(rays), capacity,
                                        ctypes.byref(launch) if launch is not None else None, stream, err, len(err))
    if st != RT_OK:
        raise RelsimError(st, err.value.decode())


def shading(**kw) -> Shading:
    """rt_shading with the reference's defaults (the sky off), overridden by keyword (field names)."""
    s = Shading()
    lib().rt_shading_defaults(ctypes.byref(s))
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def sky_profile(**fields) -> SkyProfile:
    """GpuSkyProfile's defaults with fields set by name (vector components as
    "name[k]" through a dict: sky_profile(**{"dust_tint[0]": 0.5}))."""
    p = SkyProfile()
    L = lib()
    L.rt_sky_profile_defaults(ctypes.byref(p))
    for k, v in fields.items():
        if L.rt_sky_profile_set(ctypes.byref(p), k.encode(), float(v)) != RT_OK:
            raise KeyError(k)
    return p


def sky_get(p: SkyProfile, field: str) -> float:
    v = _d()
    if lib().rt_sky_profile_get(ctypes.byref(p), field.encode(), ctypes.byref(v)) != RT_OK:
        raise KeyError(field)
    return v.value


def server_config(budget_bytes: int | None = None, record: Iterable[str] | None = None, **kw) -> ServerConfig:
    """rt_server_config with the library defaults, overridden by keyword (field names)."""
    c = ServerConfig()
    lib().rt_server_config_defaults(ctypes.byref(c))
    if budget_bytes is not None:
        c.memory_budget_bytes = int(budget_bytes)
    if record is not None:
        c.record_mask = sum(RECORD_BIT[f] for f in set(record))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class Server:
    """Continuous-batching request server (rt_server_*): submit cameras with host
    output buffers, poll finished requests.  The host buffers are kept alive here
    until their request is polled as done."""

    def __init__(self, device: int = 0, config: ServerConfig | None = None):
        L = lib()
        self.lib = L
        self.config = config if config is not None else server_config()
        h = ctypes.c_void_p()
        st = L.rt_server_create(ctypes.byref(h), device, ctypes.byref(self.config))
        if st != RT_OK:
            raise RelsimError(st, f"rt_server_create(device={device}) failed")
        self._h = h
        self._keep: dict[int, dict] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.rt_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, cam: Camera, fields: Iterable[str] = ("status", "r_hit", "g"), pixels: bool = False,
               out: dict | None = None, sources: list[Source] | None = None) -> tuple[int, dict]:
        """Queue a request (a multi-source scene when `sources` is given); returns
        (id, host arrays that receive the records).  Raises RelsimError with
        status AGAIN when the queue is full."""
        n = window_rays(cam)
        if out is None:
            out = {name: np.empty(n, dtype=dt) for name, dt in RAY_FIELDS if name in set(fields)}
            if pixels:
                out["pixels"] = np.empty(n, dtype=PIXEL_DTYPE)
        ro = RayOut()
        for name, arr in out.items():
            if name != "pixels":
                setattr(ro, name, arr.ctypes.data)
        pptr = out["pixels"].ctypes.data if "pixels" in out else None
        rid = ctypes.c_uint64()
        if sources is None:
            st = self.lib.rt_server_submit(self._h, ctypes.byref(cam), pptr, ctypes.byref(ro), n, ctypes.byref(rid))
        else:
            arr = (Source * max(len(sources), 1))(*sources)
            st = self.lib.rt_server_submit_multi(self._h, ctypes.byref(cam), arr, len(sources), pptr,
                                                 ctypes.byref(ro), n, ctypes.byref(rid))
        if st != RT_OK:
            raise RelsimError(st, self.lib.rt_server_last_error(self._h).decode() or "rt_server_submit")
        self._keep[rid.value] = out
        return rid.value, out

    def poll(self, timeout_ms: float = 0.0, max_done: int = 256) -> list[RequestDone]:
        buf = (RequestDone * max_done)()
        n = _u32()
        st = self.lib.rt_server_poll(self._h, buf, max_done, ctypes.byref(n), timeout_ms)
        if st != RT_OK:
            raise RelsimError(st, "rt_server_poll")
        done = [buf[i] for i in range(n.value)]
        for d in done:
            self._keep.pop(d.id, None)
        return done

    def set_shading(self, shading: "Shading | None") -> None:
        """Shade the pixels of requests that finish from now on (None: colour off)."""
        st = self.lib.rt_server_set_shading(self._h, ctypes.byref(shading) if shading is not None else None)
        if st != RT_OK:
            raise RelsimError(st, "rt_server_set_shading")

    def stats(self) -> ServerStats:
        s = ServerStats()
        st = self.lib.rt_server_get_stats(self._h, ctypes.byref(s))
        if st != RT_OK:
            raise RelsimError(st, "rt_server_get_stats")
        return s

    def wait(self, ids: Iterable[int], timeout_s: float = 60.0) -> dict[int, RequestDone]:
        """Poll until every id is done (or raise TimeoutError)."""
        import time

        want = set(ids)
        got: dict[int, RequestDone] = {}
        t_end = time.monotonic() + timeout_s
        while want - set(got):
            if time.monotonic() > t_end:
                raise TimeoutError(f"{len(want - set(got))} requests not done")
            for d in self.poll(timeout_ms=50.0):
                got[d.id] = d
        return got


def bundle_rays(cams: list[Camera]) -> int:
    arr = (Camera * len(cams))(*cams)
    return int(lib().rt_bundle_rays(arr, len(cams)))


def device_ray_out(n: int, fields: Iterable[str] | None = None, device: str = "cuda:0"):
    """Allocate device SoA outputs as torch tensors; returns (RayOut, {name: tensor})."""
    import torch

    tdt = {np.uint32: torch.int32, np.float64: torch.float64}
    names = [f for f, _ in RAY_FIELDS] if fields is None else list(fields)
    ro = RayOut()
    tensors = {}
    for name, dt in RAY_FIELDS:
        if name in names:
            t = torch.empty(n, dtype=tdt[dt], device=device)
            tensors[name] = t
            setattr(ro, name, t.data_ptr())
    return ro, tensors
