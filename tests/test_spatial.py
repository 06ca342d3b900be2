"""Midpoint-ordered panels (pstm_b200.spatial), the host side of the GPU
spatial query: the row ranges of a rectangle hold every trace inside it, in
ascending disjoint ranges of the sorted panel, and nothing outside its y range
or outside its two edge columns; counts and selections agree with a brute-force
scan of the rectangle (the reference's query_rectangle semantics, inclusive
bounds, spatial_index.py:178-231)."""
from __future__ import annotations

import numpy as np
import pytest

from pstm_b200.spatial import MidpointIndex, sort_panel


def _brute(mx, my, box):
    x_lo, x_hi, y_lo, y_hi = box
    return (mx >= x_lo) & (mx <= x_hi) & (my >= y_lo) & (my <= y_hi)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_runs_cover_the_rectangle_exactly(seed):
    rng = np.random.default_rng(seed)
    n = 20000
    mx = rng.uniform(0, 3000, n)
    my = rng.uniform(-500, 2500, n)
    mx[:50] = np.round(mx[:50] / 100) * 100      # midpoints on column edges
    my[50:100] = my[0]                            # ties in y
    idx = MidpointIndex(mx, my, column_width_m=100.0)
    assert sorted(idx.order.tolist()) == list(range(n))
    smx, smy = mx[idx.order], my[idx.order]
    col = np.floor((smx - idx.x0) / 100.0)
    assert np.all(np.diff(col) >= 0)
    same = np.diff(col) == 0
    assert np.all(np.diff(smy)[same] >= 0)
    tie = same & (np.diff(smy) == 0)
    assert np.all(np.diff(idx.order)[tie] > 0)    # ties keep trace order
    for _ in range(40):
        x_lo, y_lo = rng.uniform(-200, 3000), rng.uniform(-700, 2500)
        box = (x_lo, x_lo + rng.uniform(0, 1500), y_lo, y_lo + rng.uniform(0, 1500))
        if rng.random() < 0.2:                     # bounds exactly on midpoints
            j = rng.integers(0, n, 2)
            box = (min(mx[j]), max(mx[j]), min(my[j]), max(my[j]))
        runs, count = idx.runs(*box, with_count=True)
        inside = _brute(smx, smy, box)
        assert count == int(inside.sum())
        covered = np.zeros(n, bool)
        prev = 0
        for a, b in runs:
            assert prev <= a < b <= n
            prev = b
            covered[a:b] = True
        assert np.all(covered[inside])
        extra = covered & ~inside
        assert np.all((smy[extra] >= box[2]) & (smy[extra] <= box[3]))
        c_lo, c_hi = np.floor((box[0] - idx.x0) / 100.0), np.floor((box[1] - idx.x0) / 100.0)
        assert np.all((col[extra] == c_lo) | (col[extra] == c_hi))
        sel = idx.select(*box)
        np.testing.assert_array_equal(sel, np.flatnonzero(inside))


def test_empty_and_degenerate():
    idx = MidpointIndex(np.zeros(0), np.zeros(0), 50.0)
    assert idx.n_traces == 0 and idx.runs(0, 10, 0, 10).shape == (0, 2)
    idx = MidpointIndex(np.array([5.0, 15.0, 25.0]), np.array([1.0, 2.0, 3.0]), 10.0)
    assert idx.runs(100, 200, 0, 10).shape == (0, 2)          # right of every column
    assert idx.runs(-50, -20, 0, 10).shape == (0, 2)          # left of every column
    assert idx.runs(20, 10, 0, 10).shape == (0, 2)            # x_hi < x_lo
    assert idx.runs(0, 30, 5, 4).shape == (0, 2)              # y_hi < y_lo
    r, c = idx.runs(0, 30, 0, 10, with_count=True)
    np.testing.assert_array_equal(r, [[0, 3]])                # adjacent columns merge
    assert c == 3
    with pytest.raises(ValueError):
        MidpointIndex(np.array([np.nan]), np.array([0.0]), 10.0)
    with pytest.raises(ValueError):
        MidpointIndex(np.zeros(3), np.zeros(2), 10.0)
    with pytest.raises(ValueError):
        MidpointIndex(np.zeros(3), np.zeros(3), 0.0)
    with pytest.raises(ValueError):
        MidpointIndex(np.array([1.0]), np.array([1.0]), 10.0, x0=5.0)


def test_sort_panel_numpy():
    from pstm_b200 import workloads
    case = workloads.config1(n_traces=300, nx=4, ny=4, nt=20)
    tb = case.traces
    idx = MidpointIndex(tb.midpoint_x, tb.midpoint_y, 200.0)
    st = sort_panel(tb, idx)
    np.testing.assert_array_equal(st.amplitudes, tb.amplitudes[idx.order])
    np.testing.assert_array_equal(st.source_x, tb.source_x[idx.order])
    np.testing.assert_array_equal(st.midpoint_y, idx.my_sorted)
    assert st.sample_rate_ms == tb.sample_rate_ms
