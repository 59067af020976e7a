"""ctypes bindings of the CPU checker libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check in
__graft_entry__.py and by the cpu_baseline / reference legs of bench.py.  The
product (the CUDA library and its host code) never imports this module.

  liboracle.so           C restatement of the reference's FP64 null-ray paths
                         (ks_oracle.c Kerr-Schild, ms_oracle.c multi-source,
                         bl_oracle.c Boyer-Lindquist Kerr-Newman; see their
                         headers for the citations)
  _ref/libref_oracle.so  the reference's own functions, compiled from its
                         headers by oracle/Makefile (present where it was built)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_oracle.so")

CAMERA_DTYPE = np.dtype([
    ("observer_position", "f8", 4),
    ("tetrad_e1", "f8", 4),
    ("tetrad_e2", "f8", 4),
    ("tetrad_e3", "f8", 4),
    ("field_of_view_rad", "f8"),
    ("metric_mass", "f8"),
    ("metric_spin", "f8"),
    ("escape_radius", "f8"),
    ("capture_scale", "f8"),
    ("disk_inner_radius", "f8"),
    ("disk_outer_radius", "f8"),
    ("rtol", "f8"),
    ("atol", "f8"),
    ("step_cap_fraction", "f8"),
    ("initial_step_fraction", "f8"),
    ("projection_tol", "f8"),
    ("screen_width", "u4"),
    ("screen_height", "u4"),
    ("max_steps", "u4"),
    ("early_capture", "u4"),
])

RAY_DTYPE = np.dtype([
    ("status", "u4"), ("flags", "u4"), ("steps_accepted", "u4"), ("steps_rejected", "u4"),
    ("r", "f8"), ("theta", "f8"), ("phi", "f8"), ("r_hit", "f8"), ("g", "f8"), ("lambda", "f8"),
    ("dH", "f8"), ("dE", "f8"), ("dLz", "f8"), ("dQ", "f8"), ("db_shadow", "f8"), ("exit_dir", "f8", (3,)),
    ("body", "u4"), ("pad", "u4"),
])
BODY_NONE = 0xFFFFFFFF

CAPTURED, ESCAPED, DISK, UNFINISHED = 1, 2, 3, 0

# orc_cont: the translucent-disk continuation of a ray (ks_oracle.h)
MAX_CROSSINGS = 8
CONT_DTYPE = np.dtype([
    ("n_cross", "u4"), ("fate", "u4"), ("cross_r", "f8", MAX_CROSSINGS), ("cross_phi", "f8", MAX_CROSSINGS),
    ("cross_g", "f8", MAX_CROSSINGS), ("exit_dir", "f8", (3,)), ("cross_src", "u4", MAX_CROSSINGS),
    ("near_source", "u4"), ("pad", "u4"),
])

# orc_fm: the Fishbone-Moncrief torus of hydro model 2 with the resolved disk profile (ks_oracle.h)
FM_DTYPE = np.dtype([
    ("m", "f8"), ("a", "f8"), ("rh", "f8"), ("l", "f8"), ("w_in", "f8"), ("h_max", "f8"), ("inner", "f8"),
    ("outer", "f8"), ("exponent", "f8"), ("kappa", "f8"), ("density", "f8"), ("valid", "u4"), ("closed", "u4"),
    ("profile", "f4", 32),
])

# orc_source: a black-hole body beside the camera's hole (ms_oracle.c)
SOURCE_DTYPE = np.dtype([
    ("position", "f8", 3), ("mass", "f8"), ("spin_parameter", "f8"), ("axis", "f8", 3),
    ("disk_enabled", "f8"), ("disk_inner_scale", "f8"), ("disk_outer_units", "f8"),
])
MS_MAX_SOURCES = 16
MS_TABLE_DTYPE = np.dtype([
    ("count", "u4"), ("pad", "u4"), ("pos", "f8", (16, 3)), ("mass", "f8", 16), ("axis", "f8", (16, 3)),
    ("spin", "f8", 16), ("fx", "f8", (16, 3)), ("rh", "f8", 16), ("fy", "f8", (16, 3)), ("req", "f8", 16),
    ("disk_in", "f8", 16), ("disk_out", "f8", 16),
])

_D = ctypes.POINTER(ctypes.c_double)
_lib = None
_ref = None


def build(ref: bool = False) -> None:
    """Compile the checker libraries (the _ref one only where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        v = ctypes.c_void_p
        d = ctypes.c_double
        L.orc_trace.argtypes = [v, v, ctypes.c_uint64, ctypes.c_uint64, v, ctypes.c_int]
        L.orc_trace.restype = None
        L.orc_trace_cont.argtypes = [v, v, ctypes.c_uint64, ctypes.c_uint64, v, v, ctypes.c_int]
        L.orc_trace_cont.restype = None
        L.orc_ray_initial_state.argtypes = [v, ctypes.c_uint32, ctypes.c_uint32, v]
        L.orc_ray_initial_state.restype = d
        L.orc_dp45_attempt.argtypes = [v, v, d, v]
        L.orc_dp45_attempt.restype = d
        L.orc_ks_field.argtypes = [v, d, d, v, v, v]
        L.orc_ks_rhs.argtypes = [v, d, d, v]
        L.orc_ks_position_from_bl.argtypes = [d, d, d, d, v]
        L.orc_bl_from_ks.argtypes = [v, d, d, v]
        L.orc_initial_momentum.argtypes = [v, d, d, v, v]
        L.orc_isco_radius.argtypes = [d, d]
        L.orc_isco_radius.restype = d
        L.orc_redshift_at.argtypes = [d, d, d, d]
        L.orc_redshift_at.restype = d
        L.orc_pinhole_ray.argtypes = [d, d, d, v]
        L.orc_pi30_factor.argtypes = [d, d, ctypes.c_int, d]
        L.orc_pi30_factor.restype = d
        L.orc_hamiltonian.argtypes = [v, d, d]
        L.orc_hamiltonian.restype = d
        L.orc_carter_q.argtypes = [v, d, d]
        L.orc_carter_q.restype = d
        L.orc_shadow_distance.argtypes = [d, d, d, d]
        L.orc_shadow_distance.restype = d
        L.orc_ms_build.argtypes = [v, v, ctypes.c_uint32, v]
        L.orc_ms_rhs.argtypes = [v, v, v]
        L.orc_ms_hamiltonian.argtypes = [v, v]
        L.orc_ms_hamiltonian.restype = d
        L.orc_ms_initial_momentum.argtypes = [v, v, v, v]
        L.orc_ms_inside_horizon.argtypes = [v, v]
        L.orc_ms_initial_state.argtypes = [v, v, ctypes.c_uint32, ctypes.c_uint32, v]
        L.orc_ms_trace.argtypes = [v, v, v, ctypes.c_uint64, ctypes.c_uint64, v, ctypes.c_int]
        L.orc_ms_trace.restype = None
        L.orc_ms_trace_cont.argtypes = [v, v, v, ctypes.c_uint64, ctypes.c_uint64, v, v, ctypes.c_int]
        L.orc_ms_trace_cont.restype = None
        L.orc_kn_horizon.argtypes = [d, d, d]
        L.orc_kn_horizon.restype = d
        L.orc_kn_metric.argtypes = [d, d, d, d, d, v]
        L.orc_kn_metric_derivs.argtypes = [d, d, d, d, d, v, v]
        L.orc_bl_rhs.argtypes = [d, d, d, v, v]
        L.orc_bl_null_residual.argtypes = [d, d, d, v]
        L.orc_bl_null_residual.restype = d
        L.orc_bl_invariants.argtypes = [d, d, d, v, v]
        L.orc_kn_shadow_distance.argtypes = [d, d, d, d, d]
        L.orc_kn_shadow_distance.restype = d
        L.orc_bl_zamo_ray.argtypes = [d, d, d, d, d, d, d, d, v]
        L.orc_bl_initial_state.argtypes = [v, d, ctypes.c_uint32, ctypes.c_uint32, v]
        L.orc_bl_trace.argtypes = [v, d, v, ctypes.c_uint64, ctypes.c_uint64, v, ctypes.c_int]
        L.orc_bl_trace.restype = None
        L.orc_bl_trace_cont.argtypes = [v, d, v, ctypes.c_uint64, ctypes.c_uint64, v, v, ctypes.c_int]
        L.orc_bl_trace_cont.restype = None
        f = ctypes.c_float
        L.orc_planck_xyz.argtypes = [d, v]
        L.orc_blackbody_rgb.argtypes = [d, d, v]
        L.orc_resolve_profile.argtypes = [v, v, v]
        L.orc_nt_context.argtypes = [d, d, d, d, f, v]
        L.orc_disk_shade.argtypes = [v, v, ctypes.c_uint32, f, v]
        L.orc_tonemap.argtypes = [v, ctypes.c_uint32, d, v]
        L.orc_shade_cont.argtypes = [v, ctypes.c_uint32, f, ctypes.c_uint32, d, d, d, d, d, d, d, ctypes.c_uint32,
                                     v, v, v, v]
        L.orc_shade_pixel.argtypes = [v, ctypes.c_uint32, f, ctypes.c_uint32, d, d, d, d, d, d, d, ctypes.c_uint32,
                                      d, d, d, v]
        L.orc_fm_context.argtypes = [d, d, d, d, d, d, d, v, v]
        L.orc_fm_segment.argtypes = [v, v, v, d, v]
        L.orc_fm_accumulate.argtypes = [v, v, v, d, v]
        L.orc_trace_volume.argtypes = [v, v, v, ctypes.c_uint64, ctypes.c_uint64, v, v, v, ctypes.c_int]
        L.orc_bl_trace_volume.argtypes = [v, d, v, v, ctypes.c_uint64, ctypes.c_uint64, v, v, v, ctypes.c_int]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_PATH} missing: run `make -C oracle ref` where the reference tree exists")
        L = ctypes.CDLL(REF_PATH)
        v = ctypes.c_void_p
        d = ctypes.c_double
        u = ctypes.c_uint32
        L.ref_ks_field.argtypes = [v, d, d, v, v, v]
        L.ref_ks_rhs.argtypes = [v, d, d, v]
        L.ref_ks_rk4_step.argtypes = [v, d, d, d]
        L.ref_ks_position_from_bl.argtypes = [d, d, d, d, v]
        L.ref_bl_from_ks.argtypes = [v, d, d, v]
        L.ref_initial_momentum.argtypes = [v, d, d, v, v]
        L.ref_redshift_at.argtypes = [d, d, d, d]
        L.ref_redshift_at.restype = d
        L.ref_isco_radius.argtypes = [d, d]
        L.ref_isco_radius.restype = d
        L.ref_pinhole_ray.argtypes = [d, d, d, v]
        L.ref_pi30_sequence.argtypes = [v, v, ctypes.c_int, v]
        L.ref_kerr_invariants.argtypes = [v, d, d, v]
        L.ref_rk45_trace.argtypes = [v, d, d, d, d, d, d, d, d, d, ctypes.c_int, v]
        L.ref_dispatch_fp64.argtypes = [v, v, v, v, d, d, d, d, d, u, u, u, u, u, v, v, v]
        L.ref_dispatch_fp64.restype = d
        L.ref_dispatch_fp64_kn.argtypes = [v, v, v, v, d, d, d, d, d, d, u, u, u, u, u, d, v, v, v]
        L.ref_dispatch_fp64_kn.restype = d
        L.ref_ms_case.argtypes = [v, u, v, v, v, v, v, v, v, v]
        L.ref_ms_case.restype = u
        L.ref_kn_metric.argtypes = [d, d, d, v, v]
        L.ref_kerr_bl_metric.argtypes = [d, d, v, v]
        L.ref_kn_christoffel.argtypes = [d, d, d, v, v, v, v]
        L.ref_kerr_bl_christoffel.argtypes = [d, d, v, v, v, v]
        L.ref_kn_horizon.argtypes = [d, d, d]
        L.ref_kn_horizon.restype = d
        L.ref_kn_zamo_ray.argtypes = [d, d, d, d, d, d, d, d, d, v]
        L.ref_kn_rk45_trace.argtypes = [v, d, d, d, d, d, d, d, d, d, d, ctypes.c_int, v]
        L.ref_fm_context.argtypes = [v, d, d, v]
        L.ref_fm_segment.argtypes = [v, v, d, d, v, v, d, v]
        _ref = L
    return _ref


def to_camera(cam: dict) -> np.ndarray:
    """Pack a camera dict (same keys as CAMERA_DTYPE) into the C struct."""
    c = np.zeros(1, dtype=CAMERA_DTYPE)
    for name in CAMERA_DTYPE.names:
        if name in cam:
            c[name] = cam[name]
    return c


def trace(cam: dict, pixels: np.ndarray | None = None, first: int = 0, count: int | None = None,
          threads: int = 0) -> np.ndarray:
    """Trace pixels (row-major indices) through the FP64 oracle."""
    c = to_camera(cam)
    if pixels is not None:
        idx = np.ascontiguousarray(pixels, dtype=np.uint64)
        n = idx.size
        out = np.zeros(n, dtype=RAY_DTYPE)
        lib().orc_trace(_p(c), _p(idx), 0, n, _p(out), threads)
    else:
        n = int(cam["screen_width"]) * int(cam["screen_height"]) - first if count is None else count
        out = np.zeros(n, dtype=RAY_DTYPE)
        lib().orc_trace(_p(c), None, first, n, _p(out), threads)
    return out


def trace_cont(cam: dict, pixels: np.ndarray | None = None, threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Trace pixels with the translucent-disk continuation: (records of the
    first hit, as trace() gives them; CONT_DTYPE crossings and ends)."""
    c = to_camera(cam)
    if pixels is None:
        n = int(cam["screen_width"]) * int(cam["screen_height"])
        idx = None
    else:
        idx = np.ascontiguousarray(pixels, dtype=np.uint64)
        n = idx.size
    out = np.zeros(n, dtype=RAY_DTYPE)
    cont = np.zeros(n, dtype=CONT_DTYPE)
    lib().orc_trace_cont(_p(c), _p(idx) if idx is not None else None, 0, n, _p(out), _p(cont), threads)
    return out, cont


def initial_state(cam: dict, px: int, py: int) -> tuple[np.ndarray, float]:
    c = to_camera(cam)
    y = np.zeros(6)
    lz = lib().orc_ray_initial_state(_p(c), px, py, _p(y))
    return y, lz


def boundary_band(rays: np.ndarray, r_in: float, r_out: float, band: float = 1e-6) -> np.ndarray:
    """Rays within `band` M of the shadow edge (Kerr critical curve) or of a disk edge."""
    near_shadow = np.abs(rays["db_shadow"]) < band
    rh = rays["r_hit"]
    near_disk = np.isfinite(rh) & ((np.abs(rh - r_in) < band) | (np.abs(rh - r_out) < band))
    return near_shadow | near_disk


def sources_array(sources) -> np.ndarray:
    """Pack source dicts (SOURCE_DTYPE keys) into orc_source structs."""
    arr = np.zeros(len(sources), dtype=SOURCE_DTYPE)
    for i, src in enumerate(sources):
        for k in SOURCE_DTYPE.names:
            arr[i][k] = src[k]
    return arr


def ms_table(cam: dict, sources) -> np.ndarray:
    """The oracle's source table (camera hole + bodies)."""
    c = to_camera(cam)
    src = sources_array(sources)
    t = np.zeros(1, dtype=MS_TABLE_DTYPE)
    lib().orc_ms_build(_p(c), _p(src) if len(src) else None, len(src), _p(t))
    return t


def ms_trace(cam: dict, sources, pixels: np.ndarray | None = None, threads: int = 0) -> np.ndarray:
    """Trace pixels (row-major indices) of a multi-source scene through the FP64 oracle."""
    c = to_camera(cam)
    t = ms_table(cam, sources)
    if pixels is None:
        n = int(cam["screen_width"]) * int(cam["screen_height"])
        out = np.zeros(n, dtype=RAY_DTYPE)
        lib().orc_ms_trace(_p(c), _p(t), None, 0, n, _p(out), threads)
    else:
        idx = np.ascontiguousarray(pixels, dtype=np.uint64)
        out = np.zeros(idx.size, dtype=RAY_DTYPE)
        lib().orc_ms_trace(_p(c), _p(t), _p(idx), 0, idx.size, _p(out), threads)
    return out


def ms_trace_cont(cam: dict, sources, pixels: np.ndarray | None = None,
                  threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Multi-source trace with the translucent-disk continuation: (records of the
    first hits, continuation records with each crossing's source)."""
    c = to_camera(cam)
    t = ms_table(cam, sources)
    idx = None if pixels is None else np.ascontiguousarray(pixels, dtype=np.uint64)
    n = int(cam["screen_width"]) * int(cam["screen_height"]) if idx is None else idx.size
    out = np.zeros(n, dtype=RAY_DTYPE)
    cont = np.zeros(n, dtype=CONT_DTYPE)
    lib().orc_ms_trace_cont(_p(c), _p(t), None if idx is None else _p(idx), 0, n, _p(out), _p(cont), threads)
    return out, cont


def bl_initial_state(cam: dict, charge: float, px: int, py: int) -> np.ndarray:
    """Boyer-Lindquist initial state (r, theta, phi, u^t, u^r, u^theta, u^phi) of a pixel."""
    c = to_camera(cam)
    y = np.zeros(7)
    lib().orc_bl_initial_state(_p(c), charge, px, py, _p(y))
    return y


def bl_trace(cam: dict, charge: float, pixels: np.ndarray | None = None, threads: int = 0) -> np.ndarray:
    """Trace pixels (row-major indices) through the Boyer-Lindquist Kerr-Newman oracle."""
    c = to_camera(cam)
    if pixels is None:
        n = int(cam["screen_width"]) * int(cam["screen_height"])
        out = np.zeros(n, dtype=RAY_DTYPE)
        lib().orc_bl_trace(_p(c), charge, None, 0, n, _p(out), threads)
    else:
        idx = np.ascontiguousarray(pixels, dtype=np.uint64)
        out = np.zeros(idx.size, dtype=RAY_DTYPE)
        lib().orc_bl_trace(_p(c), charge, _p(idx), 0, idx.size, _p(out), threads)
    return out


def bl_trace_cont(cam: dict, charge: float, pixels: np.ndarray | None = None,
                  threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Boyer-Lindquist trace with the translucent-disk continuation: (records of
    the first hit, CONT_DTYPE crossings and ends)."""
    c = to_camera(cam)
    if pixels is None:
        n = int(cam["screen_width"]) * int(cam["screen_height"])
        idx = None
    else:
        idx = np.ascontiguousarray(pixels, dtype=np.uint64)
        n = idx.size
    out = np.zeros(n, dtype=RAY_DTYPE)
    cont = np.zeros(n, dtype=CONT_DTYPE)
    lib().orc_bl_trace_cont(_p(c), charge, _p(idx) if idx is not None else None, 0, n, _p(out), _p(cont), threads)
    return out, cont


def fm_context(mass: float, spin: float, torus: tuple, resolved_profile: np.ndarray) -> np.ndarray:
    """The oracle's torus (FM_DTYPE) for (r_in, r_center, gamma, optical_depth_scale,
    sampling_density) = torus and a resolved disk profile (32 floats)."""
    out = np.zeros(1, dtype=FM_DTYPE)
    prof = np.ascontiguousarray(resolved_profile, dtype=np.float32)
    lib().orc_fm_context(mass, spin, *[float(t) for t in torus], _p(prof), _p(out))
    return out


def fm_segment(fm: np.ndarray, frm, to, l_over_e: float) -> np.ndarray:
    """One chord through the torus: radiance r, g, b, opacity, redshift."""
    a = np.ascontiguousarray(frm, dtype=np.float64)
    b = np.ascontiguousarray(to, dtype=np.float64)
    out = np.zeros(5)
    lib().orc_fm_segment(_p(fm), _p(a), _p(b), l_over_e, _p(out))
    return out


def trace_volume(cam: dict, fm: np.ndarray, pixels: np.ndarray | None = None,
                 threads: int = 0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Trace with the torus (the camera as given: the caller turns the thin disk
    and early capture off): (records, continuation ends, gathered light [n, 6]:
    r, g, b, throughput, redshift, seen)."""
    c = to_camera(cam)
    idx = None if pixels is None else np.ascontiguousarray(pixels, dtype=np.uint64)
    n = int(cam["screen_width"]) * int(cam["screen_height"]) if idx is None else idx.size
    out = np.zeros(n, dtype=RAY_DTYPE)
    cont = np.zeros(n, dtype=CONT_DTYPE)
    vol = np.zeros((n, 6))
    lib().orc_trace_volume(_p(c), _p(fm), None if idx is None else _p(idx), 0, n, _p(out), _p(cont), _p(vol), threads)
    return out, cont, vol


def bl_trace_volume(cam: dict, charge: float, fm: np.ndarray, pixels: np.ndarray | None = None,
                    threads: int = 0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Boyer-Lindquist trace with the torus (as trace_volume)."""
    c = to_camera(cam)
    idx = None if pixels is None else np.ascontiguousarray(pixels, dtype=np.uint64)
    n = int(cam["screen_width"]) * int(cam["screen_height"]) if idx is None else idx.size
    out = np.zeros(n, dtype=RAY_DTYPE)
    cont = np.zeros(n, dtype=CONT_DTYPE)
    vol = np.zeros((n, 6))
    lib().orc_bl_trace_volume(_p(c), charge, _p(fm), None if idx is None else _p(idx), 0, n, _p(out), _p(cont),
                              _p(vol), threads)
    return out, cont, vol
