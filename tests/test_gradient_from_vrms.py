"""(v0, k) from v_rms(t) against the reference's estimate_gradient_from_vrms
(curved_ray.py:145-201), on the golden fixture made by
tests/golden/make_gradient_golden.py (short axes and sparse windows
included)."""
from __future__ import annotations

import os

import numpy as np

from pstm_b200.workloads import estimate_gradient_from_vrms

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gradient_from_vrms.npz")


def test_matches_reference_golden():
    d = np.load(FIXTURE)
    want = d["v0k"]
    for i in range(len(want)):
        got = estimate_gradient_from_vrms(d[f"v{i}"], d[f"t{i}"])
        np.testing.assert_allclose(got, want[i], rtol=1e-9, atol=1e-9)


def test_case2_velocity_law():
    t = np.arange(1500) * 2.0
    v0, k = estimate_gradient_from_vrms(1500.0 + 2500.0 * t / 3000.0, t)
    assert abs(v0 - 1500.0) < 1e-6 and abs(k - 2.0 * (2500.0 / 3.0) / 1500.0) < 1e-9
