"""Known answer: migration focuses each point diffractor at its position and
zero-offset time, as the reference's integration test expects of its
diffractor (tests/test_integration.py:124-130: the peak inside the window
around the diffractor's time).  The case-1 panel holds the responses of three
diffractors, (800, 800, 0.6 s), (500, 1100, 1.0 s) and (1200, 400, 1.4 s)
at v = 2000 m/s, plus noise at SNR 10.  Checked on the oracle (CPU) over a
9 x 9-pillar neighbourhood of each: the largest |image| sits on the
diffractor's pillar within one sample of its t0, and the pillar 100 m away
diagonally holds far less energy around t0."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle

DX, DT_MS, NT = 25.0, 4.0, 500


def neighbourhood(xd, yd):
    ix, iy = int(round(xd / DX)), int(round(yd / DX))
    return slice(ix - 4, ix + 5), slice(iy - 4, iy + 5)


def check_focus(img, t0_s):
    """img: (9, 9, nt) image around a diffractor pillar (at [4, 4])."""
    a = np.abs(img)
    px, py, pt = np.unravel_index(np.argmax(a), a.shape)
    it0 = int(round(t0_s * 1000.0 / DT_MS))
    assert (px, py) == (4, 4), f"peak at pillar offset {(px - 4, py - 4)}"
    assert abs(pt - it0) <= 1, f"peak {pt - it0} samples from t0"
    w = slice(it0 - 10, it0 + 11)
    assert (a[4, 4, w] ** 2).sum() >= 50.0 * (a[0, 0, w] ** 2).sum()


@pytest.mark.parametrize("k", range(3))
def test_oracle_focuses_the_diffractors(k):
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile
    oracle.build()
    case = workloads.config1()
    xd, yd, t0 = workloads.C1_DIFFRACTORS[k]
    xs, ys = neighbourhood(xd, yd)
    o = case.output
    sub = OutputTile(image=np.zeros((9, 9, NT)), fold=np.zeros((9, 9), np.int32), x_axis=o.x_axis[xs],
                     y_axis=o.y_axis[ys], t_axis_ms=o.t_axis_ms)
    oracle.migrate(case.traces, sub, case.velocity, case.config)
    check_focus(sub.image, t0)
