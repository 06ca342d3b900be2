"""Golden (v0, k) of the reference's ``estimate_gradient_from_vrms``
(``pstm/algorithm/curved_ray.py:145-201``) on seeded v_rms(t) functions,
including short axes and axes with fewer than two samples in the 500 ms
window.  Writes ``tests/golden/gradient_from_vrms.npz``; run where the
reference is at REF (``PSTM_REFERENCE``, default the installed reference in ``baseline/_ref``):

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_gradient_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gradient_from_vrms.npz")


def cases():
    rng = np.random.default_rng(17)
    out = []
    for _ in range(60):
        n = int(rng.integers(1, 40))
        t = np.sort(rng.uniform(0, 3000, n)) if rng.random() < 0.5 else \
            np.arange(n) * float(rng.choice([2.0, 4.0, 100.0, 400.0]))
        v = 1500 + rng.uniform(-500, 3000) * t / 3000 + rng.normal(0, 30, n)
        out.append((t, v))
    return out


def main():
    sys.dont_write_bytecode = True
    sys.path.insert(0, REF)
    from pstm.algorithm.curved_ray import estimate_gradient_from_vrms
    cs = cases()
    res = {f"t{i}": t for i, (t, _) in enumerate(cs)}
    res.update({f"v{i}": v for i, (_, v) in enumerate(cs)})
    res["v0k"] = np.array([estimate_gradient_from_vrms(v, t) for t, v in cs])
    np.savez_compressed(OUT, **res)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
