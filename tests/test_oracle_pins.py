"""Pin the C restatement (oracle/ks_oracle.c) against the reference itself.

The golden vectors in tests/golden/ were produced by the reference's own
functions (tests/golden/make_golden.py, through oracle/_ref built from the
unmodified reference headers).  These tests run on the CPU without the
reference tree.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(GOLDEN, "ref_functions.npz"))


def _p(a):
    return O._p(a)


def _rel(a, b, floor=1e-300):
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def test_ks_field_matches_reference(fx):
    L = O.lib()
    for i in range(len(fx["mass"])):
        x = np.ascontiguousarray(fx["y"][i, :3])
        r, h, k = np.zeros(1), np.zeros(1), np.zeros(3)
        L.orc_ks_field(_p(x), fx["mass"][i], fx["spin"][i], _p(r), _p(h), _p(k))
        np.testing.assert_allclose([r[0], h[0], *k], fx["field"][i], rtol=1e-13, atol=1e-15)  # FMA contraction differs


def test_hamiltonian_rhs_matches_reference(fx):
    """kerr_schild_null_derivatives (kerr_schild_null_integrator.hpp:72-114)."""
    L = O.lib()
    worst = 0.0
    for i in range(len(fx["mass"])):
        y = np.ascontiguousarray(fx["y"][i])
        d = np.zeros(6)
        L.orc_ks_rhs(_p(y), fx["mass"][i], fx["spin"][i], _p(d))
        scale = np.max(np.abs(fx["rhs"][i]))
        worst = max(worst, np.max(np.abs(d - fx["rhs"][i])) / scale)
    assert worst < 1e-13


def test_rk4_step_composes_from_rhs(fx):
    """The reference's RK4 step (kerr_schild_null_integrator.hpp:117-139) rebuilt
    from the oracle's RHS agrees to rounding: the RHS is the same function."""
    L = O.lib()
    for i in range(len(fx["mass"])):
        m, a, h = fx["mass"][i], fx["spin"][i], fx["rk4_h"][i]
        y = np.ascontiguousarray(fx["y"][i])

        def f(s):
            d = np.zeros(6)
            L.orc_ks_rhs(_p(np.ascontiguousarray(s)), m, a, _p(d))
            return d

        k1 = f(y)
        k2 = f(y + 0.5 * h * k1)
        k3 = f(y + 0.5 * h * k2)
        k4 = f(y + h * k3)
        out = y + h / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
        np.testing.assert_allclose(out, fx["rk4"][i], rtol=1e-12, atol=1e-12 * np.max(np.abs(fx["rk4"][i])))


def test_bl_ks_maps_match_reference(fx):
    L = O.lib()
    for i in range(len(fx["mass"])):
        r, th, ph = fx["bl_in"][i]
        o = np.zeros(3)
        L.orc_ks_position_from_bl(r, th, ph, fx["spin"][i], _p(o))
        np.testing.assert_allclose(o, fx["ks_pos"][i], rtol=1e-15, atol=1e-13)
        b = np.zeros(3)
        L.orc_bl_from_ks(_p(np.ascontiguousarray(fx["ks_pos"][i])), fx["spin"][i], fx["bl_prev_phi"][i], _p(b))
        np.testing.assert_allclose(b, fx["bl_out"][i], rtol=1e-14, atol=1e-13)
        # round trip recovers r and theta, phi modulo 2 pi
        assert abs(b[0] - r) < 1e-11 * r
        assert abs(b[1] - th) < 1e-9
        assert abs(np.angle(np.exp(1j * (b[2] - ph)))) < 1e-9


def test_initial_momentum_matches_reference(fx):
    """kerr_schild_initial_momentum (kerr_schild_null_integrator.hpp:142-194)."""
    L = O.lib()
    for i in range(len(fx["mass"])):
        p = np.zeros(3)
        L.orc_initial_momentum(_p(np.ascontiguousarray(fx["mom_x"][i])), fx["mass"][i], fx["spin"][i],
                               _p(np.ascontiguousarray(fx["mom_outward"][i])), _p(p))
        np.testing.assert_allclose(p, fx["mom_p"][i], rtol=1e-14, atol=1e-14)
        # the covector is null with p_t = -1
        y = np.ascontiguousarray(np.concatenate([fx["mom_x"][i], p]))
        assert abs(L.orc_hamiltonian(_p(y), fx["mass"][i], fx["spin"][i])) < 1e-12


def test_pinhole_redshift_isco_match_reference(fx):
    L = O.lib()
    for i in range(len(fx["mass"])):
        n = np.zeros(3)
        L.orc_pinhole_ray(fx["pin_uv"][i, 0], fx["pin_uv"][i, 1], fx["pin_fov"][i], _p(n))
        np.testing.assert_allclose(n, fx["pin_n"][i], rtol=1e-15, atol=1e-16)
        g = L.orc_redshift_at(fx["mass"][i], fx["spin"][i], fx["z_r"][i], fx["z_lz"][i])
        assert abs(g - fx["z_g"][i]) <= 1e-14 * abs(fx["z_g"][i])
        # NovikovThorneDisk::isco_radius vs the engine's kerr_isco_radius: same closed
        # form, different clamps of a/M beyond extremality
        if abs(fx["spin"][i]) < 0.999 * fx["mass"][i]:
            assert abs(L.orc_isco_radius(fx["mass"][i], fx["spin"][i]) - fx["isco"][i]) < 1e-12 * fx["isco"][i]


def test_isco_known_values():
    """test_novikov_thorne_disk.cpp:32-60: 6 M at a=0, in (1, 1.3) prograde a=.998,
    in (8, 9.5) retrograde a=-.9."""
    L = O.lib()
    assert abs(L.orc_isco_radius(1.0, 0.0) - 6.0) < 1e-12
    assert 1.0 < L.orc_isco_radius(1.0, 0.998) < 1.3
    assert 8.0 < L.orc_isco_radius(1.0, -0.9) < 9.5


def test_pi30_controller_sequence_matches_reference(fx):
    """AdaptiveStepController PI30 (step_controller.hpp:44-78), history included."""
    L = O.lib()
    prev, hist = 1.0, 0
    for e, k, ref in zip(fx["pi_err"], fx["pi_order"], fx["pi_factor"]):
        f = L.orc_pi30_factor(e, prev, hist, k)
        assert abs(f - ref) <= 1e-13 * abs(ref)
        prev, hist = max(e, 1e-12), 1


def test_invariants_match_reference(fx):
    """E, L_z and Carter Q of the oracle against compute_kerr_invariants_bl applied
    to the reference's own KS -> BL map (kerr_invariants.hpp:21-58, 116-155)."""
    L = O.lib()
    for i in range(len(fx["mass"])):
        y = np.ascontiguousarray(fx["inv_y"][i])
        m, a = fx["mass"][i], fx["spin"][i]
        energy, lz, q, _, norm = fx["inv"][i]
        assert abs(energy - 1.0) < 1e-9
        assert abs((y[0] * y[4] - y[1] * y[3]) - lz) < 1e-9 * max(1.0, abs(lz))
        qo = L.orc_carter_q(_p(y), m, a)
        assert abs(qo - q) < 1e-8 * max(1.0, abs(q)), (i, qo, q)
        assert abs(norm) < 1e-9


def test_shadow_distance_schwarzschild_critical_value():
    """a = 0: critical impact parameter b_c = 3 sqrt(3) M (the Bardeen/Synge value
    used by test_schwarzschild_shadow_render.cpp:24-86)."""
    L = O.lib()
    bc = 3.0 * np.sqrt(3.0)
    for xi_frac in (0.0, 0.3, 1.0):
        for db in (-1e-3, 1e-3):
            b = bc + db
            xi = xi_frac * b
            eta = b * b - xi * xi
            d = L.orc_shadow_distance(1.0, 0.0, xi, eta)
            # positive inside the shadow (b < b_c), magnitude ~ |db|
            assert np.sign(d) == -np.sign(db)
            assert abs(abs(d) - abs(db)) < 2e-2 * abs(db)
