"""The library's procedural sky (csrc/rt_sky.cuh, compiled here for the host)
against the reference's own SkyboxRenderer::sample_sky (compiled from the
reference headers into oracle/_ref): every layer and model switched on in
turn, on random directions near its features and over the whole sphere.
Same arithmetic on both sides; the bar is 1e-5 relative (max over the three
channels, with a 1e-7 floor), which leaves room for the compilers' different
contraction of the two sources."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "relativity-simulator_b200", "csrc")
PROFILE_BYTES = 1808


@pytest.fixture(scope="module")
def libs(tmp_path_factory):
    if not O.ref_available():
        pytest.skip("reference checker library not built")
    out = tmp_path_factory.mktemp("sky") / "libsky_host.so"
    subprocess.run(["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-shared", "-I", CSRC,
                    os.path.join(HERE, "sky", "sky_host.cpp"), "-o", str(out)], check=True)
    host = ctypes.CDLL(str(out))
    ref = O.ref()
    v, d = ctypes.c_void_p, ctypes.c_double
    for f in (host.host_sample_sky, ref.ref_sample_sky):
        f.argtypes = [v, d, d, d, d, d, v]
        f.restype = None
    ref.ref_sky_profile_defaults.argtypes = [v]
    host.host_sky_offset.argtypes = [ctypes.c_char_p, v]
    host.host_sky_offset.restype = ctypes.c_long
    return host, ref


def _defaults(ref):
    buf = np.zeros(PROFILE_BYTES, np.uint8)
    ref.ref_sky_profile_defaults(buf.ctypes.data)
    return buf


def _case(host, ref, **kw):
    buf = _defaults(ref)
    for k, v in kw.items():
        kind = ctypes.c_int()
        off = host.host_sky_offset(k.encode(), ctypes.byref(kind))
        assert off >= 0, k
        raw = np.float64(v).tobytes() if kind.value == 1 else np.uint32(v).tobytes()
        buf[off:off + len(raw)] = np.frombuffer(raw, np.uint8)
    return buf


ONLY = dict(stars_enabled=0, nebula_enabled=0, dust_enabled=0, galaxies_enabled=0, quasar_enabled=0,
            pulsar_enabled=0, snr_enabled=0)

CASES = {
    "defaults": {},
    **{f"stars_profile_{m}": dict(ONLY, stars_enabled=1, star_profile_model=m) for m in range(8)},
    "stars_pinpoint_wide": dict(ONLY, stars_enabled=1, star_profile_model=6, star_dirac_concentration=0.1),
    **{f"stars_placement_{m}": dict(ONLY, stars_enabled=1, star_placement_model=m) for m in range(6)},
    "stars_moving": dict(ONLY, stars_enabled=1, dynamic_motion=1, star_scintillation=0.5, time_seconds=3.0),
    "nebulae": dict(ONLY, nebula_enabled=1),
    "dust": dict(ONLY, dust_enabled=1),
    **{f"galaxies_{m}": dict(ONLY, galaxies_enabled=1, galaxy_morphology_model=m, galaxy_size_scale=4.0)
       for m in range(7)},
    **{f"clusters_{m}": dict(ONLY, clusters_enabled=1, cluster_placement_model=m, cluster_density=6.0,
                             cluster_brightness=1.0, cluster_size_scale=4.0, cluster_plane_scale_height=1.0)
       for m in range(4)},
    "quasars": dict(ONLY, quasar_enabled=1),
    "pulsars": dict(ONLY, pulsar_enabled=1),
    "remnants": dict(ONLY, snr_enabled=1, snr_density=10.0),
    "quasars_dense": dict(ONLY, quasar_enabled=1, quasar_density=10.0),
    "pulsars_dense": dict(ONLY, pulsar_enabled=1, pulsar_density=10.0, pulsar_wind_nebula_scale=0.02),
    **{f"grid_fill_{m}": dict(grid_enabled=1, grid_cell_fill_mode=m, grid_show_polar_caps=1, grid_show_equator=1,
                              grid_show_meridians=1, grid_show_ticks=1, grid_cell_color_count=5) for m in range(5)},
    "rotating_hue": dict(dynamic_rotation=1, hue_shift_deg=40.0),
}


def _dirs(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


@pytest.mark.parametrize("name", list(CASES))
def test_sky_matches_reference(libs, name):
    host, ref = libs
    prof = _case(host, ref, **CASES[name])
    fov, time = np.radians(90.0 if "pinpoint" in name else 30.0), 2.5
    dirs = _dirs(20000 if "galax" in name else 4000, sum(map(ord, name)))
    a = np.zeros(3, np.float32)
    b = np.zeros(3, np.float32)
    worst, lit, where = 0.0, 0, None
    for x, y, z in dirs:
        host.host_sample_sky(prof.ctypes.data, x, y, z, fov, time, a.ctypes.data)
        ref.ref_sample_sky(prof.ctypes.data, x, y, z, fov, time, b.ctypes.data)
        err = np.max(np.abs(a.astype(np.float64) - b) / np.maximum(np.abs(b), 1e-7))
        if err > worst:
            worst, where = float(err), (x, y, z, a.copy(), b.copy())
        lit += int(b.max() > 1e-6)
    if CASES[name].get("star_profile_model") != 6 or "wide" in name:
        assert lit > 0, "case lights no direction"
    assert worst < 1e-5, (name, worst, where)


def test_profile_accessors_write_the_reference_layout(libs):
    """rt_sky_profile_defaults gives the reference's GpuSkyProfile defaults byte
    for byte; rt_sky_profile_set/get reach each kind of field (u32, f64,
    vector component, grid cell colour) at the reference's offsets and refuse
    unknown names, out-of-range indices and negative or fractional-free
    overflow of u32 fields."""
    import relsim
    host, ref = libs
    p = relsim.sky_profile()
    assert bytes(p) == _defaults(ref).tobytes()
    q = relsim.sky_profile(star_profile_model=5, star_density=2.5, **{"dust_tint[1]": 0.25,
                                                                      "grid_cell_colors[3][2]": 0.75})
    want = _case(host, ref, star_profile_model=5, star_density=2.5)
    kind = ctypes.c_int()
    off = host.host_sky_offset(b"dust_tint", ctypes.byref(kind))
    want[off + 4:off + 8] = np.frombuffer(np.float32(0.25).tobytes(), np.uint8)
    off = host.host_sky_offset(b"grid_cell_colors", ctypes.byref(kind))
    want[off + (3 * 4 + 2) * 4:off + (3 * 4 + 3) * 4] = np.frombuffer(np.float32(0.75).tobytes(), np.uint8)
    assert bytes(q) == want.tobytes()
    assert relsim.sky_get(q, "star_profile_model") == 5.0
    assert relsim.sky_get(q, "star_density") == 2.5
    assert relsim.sky_get(q, "dust_tint[1]") == 0.25
    assert relsim.sky_get(q, "grid_cell_colors[3][2]") == 0.75
    for bad in ("no_such_field", "dust_tint[4]", "grid_cell_colors[16][0]", "star_density[0]"):
        with pytest.raises(KeyError):
            relsim.sky_profile(**{bad: 1.0})
    with pytest.raises(KeyError):
        relsim.sky_profile(star_profile_model=-1)
    sh = relsim.shading()
    assert sh.sky_enabled == 0 and bytes(sh.sky) == bytes(p)
