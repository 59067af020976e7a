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

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

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


def main() -> None:
    O.build(ref=True)
    rng = np.random.default_rng(20261203)
    np.savez_compressed(os.path.join(HERE, "ref_functions.npz"), **functions(rng))
    np.savez_compressed(os.path.join(HERE, "ref_rk45_rays.npz"), **rk45_rays(rng))
    np.savez_compressed(os.path.join(HERE, "ref_image_path.npz"), **image_path())
    print("wrote golden vectors to", HERE)


if __name__ == "__main__":
    main()
