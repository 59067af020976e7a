"""The oracle's Fishbone-Moncrief torus (hydro model 2: oracle/shade_oracle.c
orc_fm_context, orc_fm_segment) against the reference's own HydroDiskContext
(hydro_disk_shading.hpp:76-110, 173-269, compiled from its headers into
oracle/_ref): the torus constants and bounds, and the emission-absorption
integral of random chords through and near the torus, for several holes and
torus shapes.  Same arithmetic and library on both sides: bar 1e-12
relative."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference checker library not built")

TORI = [
    (1.0, 0.0, (6.0, 12.0, 4.0 / 3.0, 0.35, 2.0)),
    (1.0, 0.94, (6.0, 12.0, 1.3333334, 0.35, 2.0)),
    (1.0, -0.5, (5.0, 9.0, 5.0 / 3.0, 1.2, 4.0)),
    (2.0, 0.7, (4.0, 8.0, 1.4, 0.8, 0.5)),
    (1.0, 0.3, (8.0, 7.0, 4.0 / 3.0, 0.35, 2.0)),   # no equilibrium: r_in beyond the pressure maximum
]


def _profile():
    """The default disk profile resolved as rt_shading_defaults resolves it."""
    import relsim
    sh = relsim.shading()
    prof_in = np.frombuffer(bytes(sh.disk), np.float32).copy()
    over = np.array([sh.disk_temperature_scale_k, sh.disk_temperature_floor_k, sh.disk_color_saturation,
                     sh.disk_doppler_beaming_exponent])
    out = np.zeros(32, np.float32)
    O.lib().orc_resolve_profile(O._p(prof_in), O._p(over), O._p(out))
    return out


def _close(a, b, tol=1e-12):
    return abs(a - b) <= tol * max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("k", range(len(TORI)))
def test_torus_constants_match_reference(k):
    m, a, torus = TORI[k]
    fm = O.fm_context(m, a, torus, _profile())[0]
    ref = np.zeros(7)
    tor = np.array(torus, dtype=np.float64)
    O.ref().ref_fm_context(O._p(tor), m, a, O._p(ref))
    assert int(fm["valid"]) == int(ref[0])
    if not ref[0]:
        return
    assert int(fm["closed"]) == int(ref[1])
    for got, want in ((fm["h_max"], ref[2]), (fm["inner"], ref[3]), (fm["outer"], ref[4]), (fm["l"], ref[5]),
                      (fm["w_in"], ref[6])):
        assert _close(float(got), float(want)), (got, want)


@pytest.mark.parametrize("k", range(len(TORI)))
def test_torus_segments_match_reference(k):
    m, a, torus = TORI[k]
    prof = _profile()
    fm = O.fm_context(m, a, torus, prof)
    tor = np.array(torus, dtype=np.float64)
    rng = np.random.default_rng(k)
    r_in, r_c = torus[0] * m, torus[1] * m
    hits = 0
    for _ in range(300):
        # chords of up to 6 M about the ring of pressure maxima, some crossing the
        # torus's body, some not
        ph = rng.uniform(0.0, 2.0 * np.pi)
        c = np.array([r_c * np.cos(ph), r_c * np.sin(ph), 0.0]) + rng.normal(size=3) * abs(r_c - r_in) * np.array(
            [0.6, 0.6, 0.4])
        d = rng.normal(size=3)
        d *= rng.uniform(0.2, 6.0) * m / np.linalg.norm(d)
        frm, to = c - 0.5 * d, c + 0.5 * d
        l = float(rng.uniform(-6.0, 6.0))
        got = O.fm_segment(fm, frm, to, l)
        want = np.zeros(5)
        O.ref().ref_fm_segment(O._p(tor), O._p(prof), m, a, O._p(np.ascontiguousarray(frm)),
                               O._p(np.ascontiguousarray(to)), l, O._p(want))
        for i in range(5):
            assert _close(got[i], want[i]), (i, got, want)
        hits += got[3] > 1e-6
    assert hits > 30 if fm[0]["valid"] else hits == 0
