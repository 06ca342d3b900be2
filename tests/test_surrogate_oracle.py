"""CPU checks of the surrogate network's oracle and host logic (no GPU)."""
from __future__ import annotations

import numpy as np

from oracle import surrogate_ref as R


def test_oracle_backward_matches_finite_differences():
    """The analytic FP64 backward pass of the NumPy oracle against central
    differences of its loss (60 random parameters)."""
    from pstm_b200 import surrogate as S
    rng = np.random.default_rng(0)
    p = S.init_params(7).astype(np.float64)
    p[R.N_PARAMS - 1] = 0.3
    x = rng.uniform(-1, 1, (40, 7))
    t = rng.uniform(-1, 1, 40)
    _, g, _ = R.forward_backward(p, x, t, bf16_points=False)
    eps = 1e-6
    for i in rng.choice(p.size, 60, replace=False):
        a, b = p.copy(), p.copy()
        a[i] += eps
        b[i] -= eps
        fd = (R.forward_backward(a, x, t, False)[0] - R.forward_backward(b, x, t, False)[0]) / (2 * eps) / len(t)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.0078125, 1e-3], np.float32)
    r = R.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0                    # tie -> even (1.0)
    assert r[2] == np.float32(1.0078125)                  # above the tie rounds up
    assert abs(r[4] - 1e-3) <= 1e-3 * 2 ** -8


def test_parameter_layout_and_normalisation():
    from pstm_b200 import surrogate as S
    assert S.N_PARAMS == R.N_PARAMS == 8897
    d = S.survey_domain("anisotropic_vti", t0_max_s=3.0, h_max_m=3200.0)
    shift, scale = d.norm()
    lo = np.array([0.0, -3200, -3200, -3200, -3200, 1500 * 0.8, 0.0])
    hi = np.array([3.0, 3200, 3200, 3200, 3200, 4000 * 1.2, 0.15])
    for a, b, sh, sc in zip(lo, hi, shift, scale):
        assert abs((a - sh) * sc + 1.0) < 1e-12 and abs((b - sh) * sc - 1.0) < 1e-12
