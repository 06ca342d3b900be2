"""Planning of the streaming executor (CPU): passes cover every trace of a
tile's selection exactly once, groups fit half the pool, and pool rows map
back to the right traces."""
from __future__ import annotations

import numpy as np


def _index(n=5000, seed=2):
    from pstm_b200.spatial import MidpointIndex
    rng = np.random.default_rng(seed)
    mx, my = rng.uniform(0, 1000, n), rng.uniform(0, 800, n)
    return MidpointIndex(mx, my, 37.5), mx, my


def test_passes_cover_each_selected_trace_once():
    from pstm_b200.streaming import plan_passes
    idx, mx, my = _index()
    boxes = [(100, 400, 50, 300), (350, 900, 0, 800), (990, 1200, 700, 900), (2000, 3000, 0, 10)]
    B, S = 97, 6
    passes = plan_passes(idx, B, S, boxes)
    for ti, box in enumerate(boxes):
        want = np.concatenate([np.arange(a, b) for a, b in idx.runs(*box)] or [np.zeros(0, int)])
        got = [np.arange(a, b) for t, grp, runs in passes if t == ti for a, b in runs]
        got = np.concatenate(got) if got else np.zeros(0, int)
        np.testing.assert_array_equal(np.sort(got), want)          # every position once
        for t, grp, runs in passes:
            if t != ti:
                continue
            assert len(grp) <= S // 2
            for a, b in runs:                                     # inside the group's blocks
                assert set(range(a // B, (b - 1) // B + 1)) <= set(grp)
    assert not [p for p in passes if p[0] == 3]                   # an empty box makes no pass


def test_pool_runs_map_rows_to_their_traces():
    from pstm_b200.streaming import pool_runs
    idx, mx, my = _index()
    B = 64
    runs = idx.runs(200, 700, 100, 600)
    blocks = sorted({j for a, b in runs for j in range(a // B, (b - 1) // B + 1)})
    rng = np.random.default_rng(0)
    slots = rng.permutation(len(blocks) + 3)[:len(blocks)]
    slot_of = dict(zip(blocks, slots))
    pr = pool_runs(runs, B, slot_of)
    assert (np.diff(pr[:, 0]) > 0).all() and (pr[1:, 0] >= pr[:-1, 1]).all()   # ascending, disjoint
    block_of_slot = {s: j for j, s in slot_of.items()}
    rows = np.concatenate([np.arange(a, b) for a, b in pr])
    back = np.array([block_of_slot[r // B] * B + r % B for r in rows])
    want = np.concatenate([np.arange(a, b) for a, b in runs])
    np.testing.assert_array_equal(np.sort(back), want)


def test_overlap_of_copies_with_kernels():
    from pstm_b200.streaming import overlap_ms
    kernels = [(10.0, 20.0), (18.0, 30.0), (40.0, 50.0)]      # union [10, 30] and [40, 50]
    copies = [(0.0, 12.0), (25.0, 45.0), (50.0, 60.0), (31.0, 39.0)]
    assert overlap_ms(copies, kernels) == 2.0 + (5.0 + 5.0) + 0.0 + 0.0
    assert overlap_ms([], kernels) == 0.0
    assert overlap_ms(copies, []) == 0.0
