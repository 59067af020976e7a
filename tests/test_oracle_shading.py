"""Pin the shading restatement (oracle/shade_oracle.c) against the
reference's own shading functions on the golden vectors of
tests/golden/ref_shading.npz (made by tests/golden/make_golden.py from
oracle/_ref): the resolved disk profile (resolve_primary_profile / finalize),
thin-disk radiance and opacity for the procedural and the Novikov-Thorne
temperature models, the Novikov-Thorne flux normalisation, blackbody colour
and the four tonemapping modes.  The restatement is compiled with FMA
contraction as the reference is, so the float paths agree bit for bit.
Runs on the CPU without the reference tree."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_shading.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(GOLDEN)


def _p(a):
    return O._p(a)


def test_resolved_profile_matches_reference(fx):
    L = O.lib()
    for i in range(len(fx["overrides"])):
        out = np.zeros(32, np.float32)
        L.orc_resolve_profile(_p(np.ascontiguousarray(fx["profile_in"][i])), _p(np.ascontiguousarray(fx["overrides"][i])),
                              _p(out))
        np.testing.assert_array_equal(out, fx["profile"][i])


def test_disk_shading_matches_reference(fx):
    L = O.lib()
    for i in range(len(fx["points"])):
        out = np.zeros(4)
        L.orc_disk_shade(_p(np.ascontiguousarray(fx["profile"][i])), _p(np.ascontiguousarray(fx["points"][i])),
                         int(fx["model"][i]), float(fx["rate"][i]), _p(out))
        np.testing.assert_array_equal(out, fx["shade"][i])
    # both temperature models and the edge envelope are exercised
    assert set(fx["model"].tolist()) == {0, 1}
    assert np.any(fx["shade"][:, 3] == 0.0) and np.any(fx["shade"][:, 3] > 0.9)


def test_novikov_thorne_context_matches_reference(fx):
    L = O.lib()
    for i in range(len(fx["points"])):
        p = fx["points"][i]
        out = np.zeros(2)
        L.orc_nt_context(p[0], p[1], p[2], p[3], float(fx["rate"][i]), _p(out))
        np.testing.assert_allclose(out, fx["nt_context"][i], rtol=1e-12)


def test_blackbody_matches_reference(fx):
    L = O.lib()
    for T, ref in zip(fx["temperature"], fx["blackbody"]):
        out = np.zeros(3)
        L.orc_blackbody_rgb(T, 0.7, _p(out))
        np.testing.assert_allclose(out, ref, rtol=1e-13, atol=1e-300)


def test_tonemapping_matches_reference(fx):
    L = O.lib()
    for i in range(len(fx["rgb"])):
        for mode in range(4):
            out = np.zeros(3, np.float32)
            L.orc_tonemap(_p(np.ascontiguousarray(fx["rgb"][i])), mode, float(fx["exposure"][i]), _p(out))
            np.testing.assert_array_equal(out, fx["tonemap"][i, mode])


def test_blackbody_colour_temperature_order():
    """Physical check: a cooler blackbody is redder (R/B falls with T)."""
    L = O.lib()
    ratios = []
    for T in (2000.0, 4000.0, 6500.0, 12000.0, 30000.0):
        out = np.zeros(3)
        L.orc_blackbody_rgb(T, 1.0, _p(out))
        ratios.append(out[0] / max(out[2], 1e-300))
    assert all(a > b for a, b in zip(ratios, ratios[1:]))
