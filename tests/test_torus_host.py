"""The library's Fishbone-Moncrief torus (csrc/rt_torus.cuh, compiled here for
the host as the shading constants are built) against the oracle's
restatement (oracle/shade_oracle.c orc_fm_context, itself pinned to the
reference's HydroDiskContext by tests/test_oracle_torus.py): the validity,
closure, peak enthalpy, bounds, l and W_in of several tori, from the float
settings as rt_shading holds them.  Same formulas on both sides: bar 1e-13
relative."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "relativity-simulator_b200", "csrc")

TORI = [(1.0, 0.0, 6.0, 12.0), (1.0, 0.94, 6.0, 12.0), (1.0, -0.5, 5.0, 9.0), (2.0, 0.7, 4.0, 8.0),
        (1.0, 0.3, 8.0, 7.0), (1.0, 0.6, 6.0, 10.0), (0.5, 0.45, 7.0, 14.0)]


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    out = tmp_path_factory.mktemp("torus") / "libtorus_host.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC, os.path.join(HERE, "torus", "torus_host.cpp"),
                    "-o", str(out)], check=True)
    L = ctypes.CDLL(str(out))
    d, v = ctypes.c_double, ctypes.c_void_p
    L.host_torus.argtypes = [d, d, d, d, v]
    L.host_torus_fluid.argtypes = [d, d, d, d, d, d, v]
    return L


@pytest.mark.parametrize("k", range(len(TORI)))
def test_torus_context_matches_oracle(host, k):
    m, a, r_in, r_c = TORI[k]
    f32 = lambda x: float(np.float32(x))
    got = np.zeros(9)
    host.host_torus(m, a, f32(r_in), f32(r_c), got.ctypes.data)
    fm = O.fm_context(m, a, (r_in, r_c, 4.0 / 3.0, 0.35, 2.0), np.zeros(32, np.float32))[0]
    assert int(got[0]) == int(fm["valid"])
    if not fm["valid"]:
        return
    assert int(got[1]) == int(fm["closed"])
    for g, w in zip(got[2:9], (fm["h_max"], fm["inner"], fm["outer"], fm["l"], fm["w_in"], fm["a"], fm["rh"])):
        assert abs(g - float(w)) <= 1e-13 * max(abs(float(w)), 1e-300), (g, w)


def test_torus_fluid_is_physical(host):
    """Inside the torus the enthalpy exceeds 1 and the fluid moves forward in
    time and prograde with the torus's angular momentum; outside it is 1."""
    out = np.zeros(3)
    host.host_torus_fluid(1.0, 0.6, 6.0, 10.0, 10.0, np.pi / 2, out.ctypes.data)
    assert out[0] > 1.0 and out[1] > 1.0 and out[2] > 0.0
    host.host_torus_fluid(1.0, 0.6, 6.0, 10.0, 10.0, 0.2, out.ctypes.data)
    assert out[0] == 1.0
