"""The Dormand-Prince continuous extension used by the mixed tracer's disk
root (csrc/rt_device.cuh, DP::D*): the coefficients read from the CUDA header
give a dense output whose local error at mid-step falls as h^5 (order 4),
while the cubic Hermite interpolant alone falls as h^4.  Checked on the
Kepler problem against a fine reference integration."""
import os
import re
from fractions import Fraction

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "relativity-simulator_b200", "csrc", "rt_device.cuh")


def header_constants() -> dict:
    src = open(HEADER).read()
    out = {}
    for name, num, den in re.findall(r"\b([ABCDE]\d{1,2})\s*=\s*(-?[\d.]+)\s*/\s*([\d.]+)", src):
        out[name] = float(Fraction(num) / Fraction(den))
    return out


C = header_constants()
A = [[], [C["A21"]], [C["A31"], C["A32"]], [C["A41"], C["A42"], C["A43"]],
     [C["A51"], C["A52"], C["A53"], C["A54"]], [C["A61"], C["A62"], C["A63"], C["A64"], C["A65"]]]
B = [C["B1"], 0.0, C["B3"], C["B4"], C["B5"], C["B6"]]
D = [C["D1"], 0.0, C["D3"], C["D4"], C["D5"], C["D6"], C["D7"]]
CN = [0.0, 0.2, 0.3, 0.8, 8.0 / 9.0, 1.0]


def kepler(y):
    x, v = y[:2], y[2:]
    return np.concatenate([v, -x / np.linalg.norm(x) ** 3])


def dp_step(y, h):
    k = [kepler(y)]
    for s in range(1, 6):
        k.append(kepler(y + h * sum(a * kk for a, kk in zip(A[s], k))))
    y1 = y + h * sum(b * kk for b, kk in zip(B, k))
    k.append(kepler(y1))
    return y1, k


def dense(y0, y1, k, h, t, with_correction=True):
    d = y1 - y0
    b = h * k[0] - d
    c = d - h * k[6] - b
    e = h * sum(dj * kj for dj, kj in zip(D, k)) if with_correction else 0.0
    return y0 + t * (d + (1 - t) * (b + t * (c + (1 - t) * e)))


def reference(y0, h, t, n=4000):
    y = y0.copy()
    for _ in range(n):
        y, _k = dp_step(y, t * h / n)
    return y


def test_coefficients_sum_to_zero():
    assert abs(sum(D)) < 1e-15


def test_dense_output_is_fourth_order_and_hermite_third():
    y0 = np.array([1.0, 0.0, 0.0, 1.2])  # an eccentric Kepler orbit
    errs, herrs = [], []
    for h in (0.2, 0.1, 0.05):
        y1, k = dp_step(y0, h)
        ref = reference(y0, h, 0.5)
        errs.append(np.max(np.abs(dense(y0, y1, k, h, 0.5) - ref)))
        herrs.append(np.max(np.abs(dense(y0, y1, k, h, 0.5, with_correction=False) - ref)))
    ratios = [errs[i] / errs[i + 1] for i in range(2)]
    hratios = [herrs[i] / herrs[i + 1] for i in range(2)]
    assert all(r > 24.0 for r in ratios), ratios       # ~2^5
    assert all(12.0 < r < 20.0 for r in hratios), hratios  # ~2^4
    assert errs[-1] < herrs[-1] / 10.0
