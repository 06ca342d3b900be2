"""Time-variant sampling: windows against the reference's own module (CPU).

``tests/golden/time_windows.npz`` holds windows computed by the reference's
``pstm/algorithm/time_variant.py`` (``tests/golden/make_tv_golden.py``); the
restatement here must produce them exactly.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN
from pstm_b200 import time_variant as tvm


def _cases():
    z = np.load(os.path.join(GOLDEN, "time_windows.npz"))
    for i in range(int(z["n_cases"])):
        yield i, z[f"case{i}_args"], z[f"case{i}_table"], z[f"case{i}_windows"], float(z[f"case{i}_speedup"])


@pytest.mark.parametrize("case", list(_cases()), ids=lambda c: f"case{c[0]}")
def test_windows_match_reference(case):
    _, args, table, ref, speedup = case
    t0, t1, dt, fmin, fmax = args
    tab = tvm.FrequencyTimeTable(times_ms=list(table[0]), frequencies_hz=list(table[1]))
    w = tvm.compute_time_windows(t0, t1, dt, tab, int(fmin), int(fmax))
    got = np.array([[x.t_start_ms, x.t_end_ms, x.dt_effective_ms, x.downsample_factor, x.sample_start,
                     x.sample_end, x.f_max_hz] for x in w])
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got[:, :6], ref[:, :6])
    np.testing.assert_allclose(got[:, 6], ref[:, 6], rtol=1e-12)
    if int(fmax) == 8:
        assert tvm.estimate_speedup(t0, t1, dt, tab) == pytest.approx(speedup, rel=1e-12)


def test_factor_rules_and_table_checks():
    assert [tvm.nearest_power_of_2(n) for n in (0, 1, 2, 3, 5, 6, 7, 12, 100)] == [1, 1, 2, 2, 4, 4, 8, 8, 128]
    assert tvm.compute_downsample_factor(80.0, 2.0) == 2      # 6.25 ms Nyquist -> 3 base samples -> 2
    assert tvm.compute_downsample_factor(10.0, 2.0) == 8      # clamped at 8
    assert tvm.compute_downsample_factor(500.0, 2.0) == 1
    with pytest.raises(ValueError):
        tvm.FrequencyTimeTable(times_ms=[0, 0], frequencies_hz=[10, 10])
    with pytest.raises(ValueError):
        tvm.FrequencyTimeTable(times_ms=[0, 10], frequencies_hz=[10, -1])


def test_resample_host_is_np_interp():
    w = tvm.compute_time_windows(0.0, 998.0, 2.0, tvm.FrequencyTimeTable.default())
    tv = tvm.window_times(w)
    img = np.random.default_rng(2).standard_normal((3, 2, len(tv)))
    out = tvm.resample_to_uniform(img, w, 2.0, 500)
    np.testing.assert_array_equal(out[1, 1], np.interp(np.arange(500) * 2.0, tv, img[1, 1]))
