"""Pin the multi-source restatement (oracle/ms_oracle.c) against the
reference's own multi-source functions: the source table with its local
frames (build_multi_source_data), the superposed RHS (ms_rhs), the static
observer's initial null momentum (ms_initial_momentum) and the inside-horizon
test (ms_inside_horizon), on the golden scenes of
tests/golden/ref_multi_source.npz (made by tests/golden/make_golden.py from
oracle/_ref).  Runs on the CPU without the reference tree."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_multi_source.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(GOLDEN)


def _camera(spin):
    cam = np.zeros(1, dtype=O.CAMERA_DTYPE)
    cam["metric_mass"] = 1.0
    cam["metric_spin"] = spin
    cam["disk_inner_radius"] = 0.0  # r_ISCO, the reference's inner_radius_scale = 1
    cam["disk_outer_radius"] = 20.0
    return {k: cam[k][0] for k in O.CAMERA_DTYPE.names}


def _sources(bodies, n):
    out = []
    for b in bodies[:n]:
        out.append({"position": b[0:3], "mass": b[3], "spin_parameter": b[4], "axis": b[5:8], "disk_enabled": b[8],
                    # the reference carries these two as float32 (GpuDiskProfile)
                    "disk_inner_scale": float(np.float32(b[9])), "disk_outer_units": float(np.float32(b[10]))})
    return out


def _table(fx, c):
    return O.ms_table(_camera(fx["spin"][c]), _sources(fx["bodies"][c], int(fx["n_bodies"][c])))


def test_source_table_matches_reference(fx):
    for c in range(len(fx["spin"])):
        t = _table(fx, c)[0]
        n = int(fx["count"][c])
        assert t["count"] == n
        ref = fx["table"][c][:n]
        np.testing.assert_allclose(t["pos"][:n], ref[:, 0:3], rtol=0, atol=0)
        np.testing.assert_allclose(t["mass"][:n], ref[:, 3], rtol=1e-15)
        np.testing.assert_allclose(t["axis"][:n], ref[:, 4:7], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(t["spin"][:n], ref[:, 7], rtol=1e-14)
        np.testing.assert_allclose(t["fx"][:n], ref[:, 8:11], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(t["rh"][:n], ref[:, 11], rtol=1e-14)
        np.testing.assert_allclose(t["fy"][:n], ref[:, 12:15], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(t["req"][:n], ref[:, 15], rtol=1e-14)
        np.testing.assert_allclose(t["disk_in"][:n], ref[:, 16], rtol=1e-13)
        np.testing.assert_allclose(t["disk_out"][:n], ref[:, 17], rtol=1e-13)


def test_superposed_rhs_matches_reference(fx):
    worst = 0.0
    for c in range(len(fx["spin"])):
        if fx["inside"][c]:
            continue
        t = _table(fx, c)
        y = np.concatenate([fx["x"][c], fx["p"][c]])
        dy = np.zeros(6)
        O.lib().orc_ms_rhs(O._p(t), O._p(y), O._p(dy))
        ref = fx["rhs"][c]
        worst = max(worst, float(np.max(np.abs(dy - ref)) / np.max(np.abs(ref))))
    assert worst < 1e-12, worst


def test_initial_momentum_matches_reference(fx):
    worst = 0.0
    for c in range(len(fx["spin"])):
        if fx["inside"][c]:
            continue
        t = _table(fx, c)
        p = np.zeros(3)
        O.lib().orc_ms_initial_momentum(O._p(t), O._p(np.ascontiguousarray(fx["x"][c])),
                                        O._p(np.ascontiguousarray(fx["outward"][c])), O._p(p))
        worst = max(worst, float(np.max(np.abs(p - fx["p0"][c])) / np.max(np.abs(fx["p0"][c]))))
    assert worst < 1e-12, worst


def test_inside_horizon_matches_reference(fx):
    got = [O.lib().orc_ms_inside_horizon(O._p(_table(fx, c)), O._p(np.ascontiguousarray(fx["x"][c])))
           for c in range(len(fx["spin"]))]
    assert got == list(fx["inside"])
    assert 0 < sum(got) < len(got)


def test_superposed_flow_conserves_its_hamiltonian(fx):
    """The summed RHS is the Hamiltonian flow of H = (|p|^2 - 1)/2 - sum_i H_i s_i^2:
    dH/dlambda = grad_x H . dx/dl + grad_p H . dp/dl = 0 along it (finite differences)."""
    c = next(i for i in range(len(fx["spin"])) if not fx["inside"][i])
    t = _table(fx, c)
    y = np.concatenate([fx["x"][c], fx["p"][c]])
    dy = np.zeros(6)
    O.lib().orc_ms_rhs(O._p(t), O._p(y), O._p(dy))
    eps = 1e-6
    Hp = O.lib().orc_ms_hamiltonian(O._p(t), O._p(y + eps * dy))
    Hm = O.lib().orc_ms_hamiltonian(O._p(t), O._p(y - eps * dy))
    assert abs(Hp - Hm) / (2 * eps) < 1e-8 * max(1.0, np.max(np.abs(dy)))
