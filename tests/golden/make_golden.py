"""Generate the golden vectors under tests/golden/ from the reference itself.

Runs the reference's own functions through oracle/_ref/libref_oracle.so (built
from the unmodified reference headers by `make -C oracle ref`).  The outputs are
committed so that the pins run without the reference tree:

  ref_functions.npz   function-level vectors: KS field, Hamiltonian RHS, RK4
                      step, BL<->KS maps, initial momentum, pinhole ray,
                      redshift, ISCO, PI30 controller sequence, Kerr invariants
  ref_rk45_rays.npz   rays traced by the reference's RK45AdaptiveIntegrator
                      (4-D Christoffel form) from the C restatement's initial
                      states, for three camera configurations
  ref_image_path.npz  per-pixel status/iterations of the reference's CPU image
                      path (SoftwareComputeEngine::dispatch_fp64) on a 32x32
                      Kerr-Schild camera
  ref_multi_source.npz  multi-source scenes: the reference's source table
                      (build_multi_source_data), superposed RHS (ms_rhs),
                      initial momentum (ms_initial_momentum) and inside-horizon
                      answer (ms_inside_horizon) at random points
  ref_bl_image_path.npz  per-pixel status/iterations/redshift of the reference's
                      CPU image path for a Kerr-Newman camera (metric type 5,
                      trace_exact_photon, heuristic RK4) at its shipped step and
                      at 1/4 and 1/20 of it, 64x64
  ref_shading.npz     pixel shading tail: the reference's resolved disk profile
                      (resolve_primary_profile), thin-disk shading for both
                      temperature models (AccretionDiskModel::shade,
                      HydroDiskShader Novikov-Thorne context), blackbody colour
                      and apply_tonemapping on random inputs
  ref_boyer_lindquist.npz  Boyer-Lindquist Kerr-Newman form: the reference's
                      metric tensor, analytic Christoffel symbols and their
                      contraction -Gamma u u (KerrNewmanMetric and KerrMetric),
                      outer horizon and ZAMO light ray at random points, and
                      rays traced by RK45AdaptiveIntegrator<KerrNewmanMetric>
                      from the C restatement's initial states

Usage:  python tests/golden/make_golden.py [name ...]   (default: every file)
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "relativity-simulator_b200"))

from oracle import oracle as O  # noqa: E402
from cameras import config_camera  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def _p(a):
    return O._p(a)


def functions(rng: np.random.Generator) -> dict:
    R = O.ref()
    n = 256
    out: dict[str, np.ndarray] = {}
    spins = rng.uniform(-0.998, 0.998, n)
    spins[:8] = [0.0, 0.94, 0.998, -0.9, 0.5, 0.0, 0.94, 0.998]
    masses = rng.uniform(0.5, 2.0, n)
    masses[:8] = 1.0
    # positions away from the ring singularity, momenta of order 1
    rad = np.exp(rng.uniform(np.log(1.5), np.log(800.0), n))
    th = np.arccos(rng.uniform(-1, 1, n))
    ph = rng.uniform(-np.pi, np.pi, n)
    x = np.stack([rad * np.sin(th) * np.cos(ph), rad * np.sin(th) * np.sin(ph), rad * np.cos(th)], 1)
    p = rng.normal(size=(n, 3))
    y = np.concatenate([x, p], 1)
    out["mass"], out["spin"], out["y"] = masses, spins, y

    field = np.zeros((n, 5))
    rhs = np.zeros((n, 6))
    rk4 = np.zeros((n, 6))
    h_rk4 = rng.uniform(-0.5, -0.01, n)
    for i in range(n):
        r, h, k = np.zeros(1), np.zeros(1), np.zeros(3)
        xi = np.ascontiguousarray(y[i, :3])
        R.ref_ks_field(_p(xi), masses[i], spins[i], _p(r), _p(h), _p(k))
        field[i] = [r[0], h[0], *k]
        yi = np.ascontiguousarray(y[i])
        d = np.zeros(6)
        R.ref_ks_rhs(_p(yi), masses[i], spins[i], _p(d))
        rhs[i] = d
        s = yi.copy()
        R.ref_ks_rk4_step(_p(s), h_rk4[i], masses[i], spins[i])
        rk4[i] = s
    out["field"], out["rhs"], out["rk4_h"], out["rk4"] = field, rhs, h_rk4, rk4

    # BL -> KS -> BL round trip inputs
    bl_in = np.stack([rad, th, ph], 1)
    ks = np.zeros((n, 3))
    bl = np.zeros((n, 3))
    prev = ph + rng.normal(scale=0.3, size=n)
    for i in range(n):
        o = np.zeros(3)
        R.ref_ks_position_from_bl(rad[i], th[i], ph[i], spins[i], _p(o))
        ks[i] = o
        b = np.zeros(3)
        R.ref_bl_from_ks(_p(np.ascontiguousarray(o)), spins[i], prev[i], _p(b))
        bl[i] = b
    out["bl_in"], out["ks_pos"], out["bl_prev_phi"], out["bl_out"] = bl_in, ks, prev, bl

    # initial momentum from random unit outward directions at observer-like radii
    robs = np.exp(rng.uniform(np.log(5.0), np.log(500.0), n))
    x0 = np.zeros((n, 3))
    outward = rng.normal(size=(n, 3))
    outward /= np.linalg.norm(outward, axis=1, keepdims=True)
    mom = np.zeros((n, 3))
    for i in range(n):
        o = np.zeros(3)
        R.ref_ks_position_from_bl(robs[i], th[i], ph[i], spins[i], _p(o))
        x0[i] = o
        m = np.zeros(3)
        R.ref_initial_momentum(_p(o), masses[i], spins[i], _p(np.ascontiguousarray(outward[i])), _p(m))
        mom[i] = m
    out["mom_x"], out["mom_outward"], out["mom_p"] = x0, outward, mom

    uv = rng.uniform(-1.5, 1.5, (n, 2))
    fov = rng.uniform(np.radians(5), np.radians(80), n)
    pin = np.zeros((n, 3))
    for i in range(n):
        o = np.zeros(3)
        R.ref_pinhole_ray(uv[i, 0], uv[i, 1], fov[i], _p(o))
        pin[i] = o
    out["pin_uv"], out["pin_fov"], out["pin_n"] = uv, fov, pin

    rr = rng.uniform(1.0, 30.0, n)
    lz = rng.uniform(-8.0, 8.0, n)
    out["z_r"], out["z_lz"] = rr, lz
    out["z_g"] = np.array([R.ref_redshift_at(masses[i], spins[i], rr[i], lz[i]) for i in range(n)])
    out["isco"] = np.array([R.ref_isco_radius(masses[i], spins[i]) for i in range(n)])

    errs = np.exp(rng.uniform(np.log(1e-6), np.log(50.0), 64))
    errs[5] = 0.0
    orders = np.where(rng.uniform(size=64) < 0.7, 5.0, 4.0)
    fac = np.zeros(64)
    R.ref_pi30_sequence(_p(errs), _p(orders), 64, _p(fac))
    out["pi_err"], out["pi_order"], out["pi_factor"] = errs, orders, fac

    # Kerr invariants of null states (p_t = -1) built by the reference's momentum map
    inv = np.zeros((n, 5))
    null_y = np.concatenate([x0, mom], 1)
    for i in range(n):
        o = np.zeros(5)
        R.ref_kerr_invariants(_p(np.ascontiguousarray(null_y[i])), masses[i], spins[i], _p(o))
        inv[i] = o
    out["inv_y"], out["inv"] = null_y, inv
    return out


def rk45_rays(rng: np.random.Generator) -> dict:
    """Sample rays of C1/C2/C3-like cameras, traced by the reference's RK45 class."""
    R = O.ref()
    out = {}
    for tag, side in (("c1", 64), ("c2", 64), ("c3", 64)):
        cam = config_camera(tag, width=side, height=side)
        n = 48
        pix = rng.choice(side * side, n, replace=False).astype(np.uint64)
        y0 = np.zeros((n, 6))
        res = np.zeros((n, 7))
        m, a = cam["metric_mass"], cam["metric_spin"]
        r_in = O.lib().orc_isco_radius(m, a)
        for i, q in enumerate(pix):
            y, _ = O.initial_state(cam, int(q % side), int(q // side))
            y0[i] = y
            o = np.zeros(7)
            R.ref_rk45_trace(_p(y), m, a, 1e-11, 1e-12, cam["step_cap_fraction"], cam["capture_scale"],
                             cam["escape_radius"], r_in, cam["disk_outer_radius"], 200000, _p(o))
            res[i] = o
        out[f"{tag}_pixels"] = pix
        out[f"{tag}_y0"] = y0
        out[f"{tag}_res"] = res
    return out


def image_path() -> dict:
    R = O.ref()
    cam = config_camera("c2", width=32, height=32)
    W = H = 32
    st = np.zeros(W * H, np.uint32)
    it = np.zeros(W * H, np.uint32)
    z = np.zeros(W * H, np.float32)
    obs = np.ascontiguousarray(cam["observer_position"], dtype=np.float64)
    e1 = np.ascontiguousarray(cam["tetrad_e1"], dtype=np.float64)
    e2 = np.ascontiguousarray(cam["tetrad_e2"], dtype=np.float64)
    e3 = np.ascontiguousarray(cam["tetrad_e3"], dtype=np.float64)
    R.ref_dispatch_fp64(_p(obs), _p(e1), _p(e2), _p(e3), cam["field_of_view_rad"], cam["metric_mass"],
                        cam["metric_spin"], cam["escape_radius"], cam["disk_outer_radius"], W, H, 20000, 0, 0,
                        _p(st), _p(it), _p(z))
    return {"status_flags": st, "iterations": it, "redshift": z, "width": np.array(W), "height": np.array(H)}


def multi_source(rng: np.random.Generator, cases: int = 40) -> dict:
    """Random scenes of 1..15 bodies beside a camera hole; per scene one point."""
    R = O.ref()
    spins, bodies, counts, xs, ps, outs = [], [], [], [], [], []
    tables, rhs, p0, inside = [], [], [], []
    for c in range(cases):
        a = rng.uniform(0.0, 0.99)
        n = int(rng.integers(1, 16))
        b = np.zeros((15, 11))
        for i in range(n):
            b[i, 0:3] = rng.uniform(-30.0, 30.0, 3)
            b[i, 3] = rng.uniform(0.2, 1.0)
            b[i, 4] = rng.uniform(-0.95, 0.95)
            ax = rng.normal(size=3)
            b[i, 5:8] = ax / np.linalg.norm(ax) * rng.uniform(0.5, 2.0)  # not normalised: the reference normalises
            b[i, 8] = 1.0 if rng.uniform() < 0.7 else 0.0
            b[i, 9] = rng.uniform(1.0, 1.5)
            b[i, 10] = rng.uniform(8.0, 24.0)
        if c % 5 == 0:
            b[0, 5:8] = [0.0, 0.0, 2.0]  # an axis near +z takes the other helper vector
        # a point away from the holes, or (every 4th case) inside one
        x = rng.uniform(-40.0, 40.0, 3)
        if c % 4 == 3:
            x = b[0, 0:3] + 0.3 * b[0, 3] * rng.normal(size=3) / np.sqrt(3)
        pd = rng.normal(size=3)
        pd /= np.linalg.norm(pd)
        ow = rng.normal(size=3)
        ow /= np.linalg.norm(ow)
        prim = np.array([1.0, a, 1.0, 20.0])
        tab = np.zeros((16, 20))
        r6 = np.zeros(6)
        m0 = np.zeros(3)
        ins = ctypes.c_int(0)
        cnt = R.ref_ms_case(_p(prim), n, _p(b), _p(x), _p(pd), _p(ow), _p(tab), _p(r6), _p(m0), ctypes.byref(ins))
        spins.append(a)
        bodies.append(b)
        counts.append(cnt)
        xs.append(x)
        ps.append(pd)
        outs.append(ow)
        tables.append(tab)
        rhs.append(r6)
        p0.append(m0)
        inside.append(ins.value)
    return {"spin": np.array(spins), "bodies": np.array(bodies), "n_bodies": np.array([int(np.count_nonzero(bb[:, 3])) for bb in bodies]),
            "count": np.array(counts), "x": np.array(xs), "p": np.array(ps), "outward": np.array(outs),
            "table": np.array(tables), "rhs": np.array(rhs), "p0": np.array(p0), "inside": np.array(inside)}


BL_CAMERAS = {
    # tag: (spin, charge, camera keywords)
    "kn": (0.9, 0.3, dict(r_obs=50.0, incl_deg=75.0, fov_deg=30.0)),
    "kerr": (0.94, 0.0, dict(r_obs=100.0, incl_deg=17.0, fov_deg=12.0)),
    "schw": (0.0, 0.0, dict(r_obs=50.0, incl_deg=60.0, fov_deg=30.0, disk_inner=6.0)),
    "kn_hi_q": (0.5, 0.7, dict(r_obs=50.0, incl_deg=85.0, fov_deg=30.0)),
}


def boyer_lindquist(rng: np.random.Generator) -> dict:
    """Function-level vectors at random points and reference RK45 rays."""
    import relsim

    R = O.ref()
    n = 256
    out: dict[str, np.ndarray] = {}
    m = rng.uniform(0.5, 2.0, n)
    m[:8] = 1.0
    a = rng.uniform(-0.99, 0.99, n) * m
    q = rng.uniform(0.0, 1.0, n) * np.sqrt(np.maximum(m * m - a * a, 0.0)) * 0.99
    q[::3] = 0.0
    rh = np.array([R.ref_kn_horizon(m[i], a[i], q[i]) for i in range(n)])
    r = rh * 1.01 + rng.exponential(10.0, n) * m
    th = rng.uniform(0.01, np.pi - 0.01, n)
    th[:4] = [np.pi / 2, 0.02, np.pi - 0.02, 1.0]
    ph = rng.uniform(-np.pi, np.pi, n)
    u = rng.normal(size=(n, 4))
    nd = rng.normal(size=(n, 3))
    nd /= np.linalg.norm(nd, axis=1, keepdims=True)
    g = np.zeros((n, 16))
    gam = np.zeros((n, 64))
    acc = np.zeros((n, 4))
    acc_kerr = np.full((n, 4), np.nan)
    zamo = np.zeros((n, 4))
    for i in range(n):
        x = np.array([0.0, r[i], th[i], ph[i]])
        R.ref_kn_metric(m[i], a[i], q[i], _p(x), _p(g[i]))
        ui = np.ascontiguousarray(u[i])
        R.ref_kn_christoffel(m[i], a[i], q[i], _p(x), _p(ui), _p(gam[i]), _p(acc[i]))
        if q[i] == 0.0:
            R.ref_kerr_bl_christoffel(m[i], a[i], _p(x), _p(ui), None, _p(acc_kerr[i]))
        R.ref_kn_zamo_ray(m[i], a[i], q[i], r[i], th[i], ph[i], nd[i, 0], nd[i, 1], nd[i, 2], _p(zamo[i]))
    out.update(mass=m, spin=a, charge=q, rh=rh, r=r, theta=th, phi=ph, u=u, n=nd, metric=g, gamma=gam, acc=acc,
               acc_kerr=acc_kerr, zamo=zamo)
    L = O.lib()
    for tag, (spin, charge, kw) in BL_CAMERAS.items():
        side = 32
        cam = relsim.camera_dict(relsim.make_camera(spin=spin, width=side, height=side, **kw))
        k = 40
        pix = rng.choice(side * side, k, replace=False).astype(np.uint64)
        y0 = np.zeros((k, 7))
        res = np.zeros((k, 7))
        r_in = cam["disk_inner_radius"] if cam["disk_inner_radius"] > 0 else L.orc_isco_radius(1.0, spin)
        for i, pq in enumerate(pix):
            y0[i] = O.bl_initial_state(cam, charge, int(pq % side), int(pq // side))
            R.ref_kn_rk45_trace(_p(y0[i]), 1.0, spin, charge, 1e-11, 1e-12, cam["step_cap_fraction"],
                                cam["capture_scale"], cam["escape_radius"], r_in, cam["disk_outer_radius"], 200000,
                                _p(res[i]))
        out[f"{tag}_pixels"] = pix
        out[f"{tag}_y0"] = y0
        out[f"{tag}_res"] = res
    return out


BL_IMAGE_CAMERA = dict(spin=0.9, charge=0.3, r_obs=50.0, incl_deg=75.0, fov_deg=30.0, side=64)


def bl_image_path() -> dict:
    import relsim

    R = O.ref()
    c = BL_IMAGE_CAMERA
    W = c["side"]
    cam = relsim.camera_dict(relsim.make_camera(spin=c["spin"], r_obs=c["r_obs"], incl_deg=c["incl_deg"],
                                                fov_deg=c["fov_deg"], width=W, height=W,
                                                metric_form=relsim.METRIC_BOYER_LINDQUIST, charge=c["charge"]))
    obs, e1, e2, e3 = (np.ascontiguousarray(cam[k], dtype=np.float64)
                       for k in ("observer_position", "tetrad_e1", "tetrad_e2", "tetrad_e3"))
    out = {"step_scale": np.array([1.0, 0.25, 0.05])}
    for i, sc in enumerate(out["step_scale"]):
        st = np.zeros(W * W, np.uint32)
        it = np.zeros(W * W, np.uint32)
        z = np.zeros(W * W, np.float32)
        R.ref_dispatch_fp64_kn(_p(obs), _p(e1), _p(e2), _p(e3), cam["field_of_view_rad"], 1.0, c["spin"], c["charge"],
                               1000.0, 20.0, W, W, 200000, 0, 0, float(sc), _p(st), _p(it), _p(z))
        out[f"status_flags_{i}"] = st
        out[f"iterations_{i}"] = it
        out[f"redshift_{i}"] = z
    return out


DISK_PROFILE_DEFAULT = [1.0, 1.0, 24.0, 9500.0, 1200.0, 0.75, 1.0, 2.0, 0.45, 1.0, 0.0, 1.0, 1.0, 1.0, 1.0, 4.0,
                        0.35, 9.0, 3.0, 2.0, 1.2, 0.25, 0.45, 5.0, 4.0, 3.0, 0.2, 40.0, 1.0, 1.0, 1.0, 1.0]


def shading(rng: np.random.Generator, n: int = 400) -> dict:
    R = O.ref()
    f32, f64, u32 = ctypes.c_float, ctypes.c_double, ctypes.c_uint32
    v = ctypes.c_void_p
    R.ref_resolve_profile.argtypes = [v, v, v]
    R.ref_disk_shade.argtypes = [v, v, u32, f32, v]
    R.ref_nt_context.argtypes = [f64, f64, f64, f64, f32, v]
    R.ref_blackbody_rgb.argtypes = [f64, f64, v]
    R.ref_tonemap.argtypes = [v, u32, f64, v]
    base = np.array(DISK_PROFILE_DEFAULT, np.float32)
    prof = np.tile(base, (n, 1))
    prof[1::2] *= rng.uniform(0.5, 1.5, (n // 2, 32)).astype(np.float32)
    prof[1::2, 24] = rng.integers(1, 7, n // 2)
    over = np.stack([rng.uniform(3000, 50000, n), rng.uniform(0, 3000, n), rng.uniform(0.5, 1.5, n),
                     rng.uniform(0, 6, n)], 1)
    over[0] = [23796.0, 1200.0, 1.0, 5.32]  # the push constants' defaults
    resolved = np.zeros((n, 32), np.float32)
    points = np.zeros((n, 9))
    model = (np.arange(n) % 2).astype(np.uint32)
    rate = (1.0 + np.arange(n) % 3).astype(np.float32)
    shade = np.zeros((n, 4))
    ntc = np.zeros((n, 2))
    for i in range(n):
        R.ref_resolve_profile(_p(prof[i]), _p(over[i]), _p(resolved[i]))
        spin = rng.uniform(-0.99, 0.99)
        inner = rng.uniform(1.5, 7.0)
        outer = rng.uniform(inner * 1.1, 40.0)
        points[i] = [1.0, spin, inner, outer, rng.uniform(inner * 0.9, outer * 1.1), rng.uniform(-20, 20),
                     rng.uniform(0.2, 2.5), rng.uniform(0, 50), rng.uniform(0, 1)]
        R.ref_disk_shade(_p(resolved[i]), _p(points[i]), int(model[i]), float(rate[i]), _p(shade[i]))
        R.ref_nt_context(1.0, spin, inner, outer, float(rate[i]), _p(ntc[i]))
    temps = np.exp(rng.uniform(np.log(200.0), np.log(5e5), n))
    bb = np.zeros((n, 3))
    for i in range(n):
        R.ref_blackbody_rgb(temps[i], 0.7, _p(bb[i]))
    rgb = rng.exponential(0.5, (n, 3))
    rgb[:4] = 0.0
    ev = rng.uniform(-2, 2, n)
    tone = np.zeros((n, 4, 3), np.float32)
    for i in range(n):
        for mode in range(4):
            R.ref_tonemap(_p(rgb[i]), mode, ev[i], _p(tone[i, mode]))
    return {"profile_in": prof, "overrides": over, "profile": resolved, "points": points, "model": model,
            "rate": rate, "shade": shade, "nt_context": ntc, "temperature": temps, "blackbody": bb, "rgb": rgb,
            "exposure": ev, "tonemap": tone}


def main() -> None:
    O.build(ref=True)
    rng = np.random.default_rng(20261203)
    makers = {
        "ref_functions": lambda: functions(rng),
        "ref_rk45_rays": lambda: rk45_rays(rng),
        "ref_image_path": image_path,
        "ref_multi_source": lambda: multi_source(np.random.default_rng(12)),
        "ref_boyer_lindquist": lambda: boyer_lindquist(np.random.default_rng(5)),
        "ref_bl_image_path": bl_image_path,
        "ref_shading": lambda: shading(np.random.default_rng(9)),
    }
    wanted = sys.argv[1:] or list(makers)
    for name in makers:  # in this order: the first two share one generator
        if name in wanted or (name == "ref_functions" and "ref_rk45_rays" in wanted):
            data = makers[name]()
            if name in wanted:
                np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
    print("wrote golden vectors to", HERE)


if __name__ == "__main__":
    main()
