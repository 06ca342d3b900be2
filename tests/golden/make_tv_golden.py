"""Golden time windows from the reference's own time-variant module.

Runs ``compute_time_windows`` of ``pstm/algorithm/time_variant.py`` (pure
Python + SciPy PCHIP) from the reference checkout and stores the windows of a
few tables and time ranges in ``tests/golden/time_windows.npz``.  Run once in a
container that has the reference at REF (``PSTM_REFERENCE``, default the installed reference in ``baseline/_ref``):

    python tests/golden/make_tv_golden.py
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")
HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # (t_min_ms, t_max_ms, base_dt_ms, table pairs, min_factor, max_factor)
    (0.0, 3998.0, 2.0, None, 1, 8),
    (0.0, 1996.0, 4.0, None, 1, 8),
    (100.0, 2998.0, 2.0, [(0, 120), (800, 70), (2000, 30), (3000, 18)], 1, 8),
    (0.0, 5998.0, 2.0, [(0, 50), (6000, 10)], 1, 16),
    (0.0, 998.0, 1.0, [(0, 400), (1000, 300)], 1, 8),
]


def main():
    spec = importlib.util.spec_from_file_location("tv_reference", os.path.join(REF, "pstm/algorithm/time_variant.py"))
    m = importlib.util.module_from_spec(spec)
    sys.modules["tv_reference"] = m
    spec.loader.exec_module(m)
    out = {}
    for i, (t0, t1, dt, pairs, fmin, fmax) in enumerate(CASES):
        table = m.FrequencyTimeTable.default() if pairs is None else m.FrequencyTimeTable.from_list(pairs)
        w = m.compute_time_windows(t0, t1, dt, table, fmin, fmax)
        out[f"case{i}_args"] = np.array([t0, t1, dt, fmin, fmax])
        out[f"case{i}_table"] = np.array([table.times_ms, table.frequencies_hz])
        out[f"case{i}_windows"] = np.array([[x.t_start_ms, x.t_end_ms, x.dt_effective_ms, x.downsample_factor,
                                              x.sample_start, x.sample_end, x.f_max_hz] for x in w])
        out[f"case{i}_speedup"] = np.array(m.estimate_speedup(t0, t1, dt, table))
    np.savez(os.path.join(HERE, "time_windows.npz"), n_cases=len(CASES), **out)


if __name__ == "__main__":
    main()
