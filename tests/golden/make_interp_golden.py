"""Golden values of the reference's trace interpolators.

Calls ``interpolate_sample`` of ``pstm/kernels/interpolation.py`` (Numba) from
the reference checkout for every method on seeded traces and sample
positions (including the trace ends, where the higher-order methods fall back
to linear) and stores them in ``tests/golden/interp_methods.npz``.  Run once in
a container that has the reference at REF (``PSTM_REFERENCE``, default the installed reference in ``baseline/_ref``):

    NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_interp_golden.py
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")
HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's method codes (interpolation.py:293-301)
METHODS = {"nearest": 0, "linear": 1, "cubic": 2, "sinc4": 3, "sinc8": 4, "sinc16": 5, "lanczos3": 6, "lanczos5": 7}


def main():
    sys.path.insert(0, REF)
    spec = importlib.util.spec_from_file_location("interp_reference",
                                                  os.path.join(REF, "pstm/kernels/interpolation.py"))
    m = importlib.util.module_from_spec(spec)
    sys.modules["interp_reference"] = m
    spec.loader.exec_module(m)
    rng = np.random.default_rng(11)
    n = 48
    traces = rng.standard_normal((6, n))
    ts = np.concatenate([rng.uniform(0, n - 1, 60), [0.0, 0.3, 1.0, 1.7, 2.5, 3.9, 4.0, n - 9.2, n - 5.5,
                                                        n - 4.0, n - 3.2, n - 2.0, n - 1.5, n - 1.0, 7.0, 12.5]])
    out = np.zeros((len(METHODS), traces.shape[0], len(ts)))
    for name, code in METHODS.items():
        for i, tr in enumerate(traces):
            for j, t in enumerate(ts):
                out[code, i, j] = m.interpolate_sample(tr, float(t), code)
    np.savez(os.path.join(HERE, "interp_methods.npz"), traces=traces, t_samples=ts, values=out,
             method_names=np.array(list(METHODS)), reference_codes=np.array(list(METHODS.values())))


if __name__ == "__main__":
    main()
