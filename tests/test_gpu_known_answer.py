"""Known answer on the CUDA path: the full case-1 tile (64 x 64 x 500 against
16,384 traces) migrated by the backend focuses each of the three diffractors
on its pillar within one sample of its t0 (the checks of
tests/test_known_answer.py, on the product path)."""
from __future__ import annotations

import pytest

from test_known_answer import check_focus, neighbourhood

pytestmark = pytest.mark.gpu


def test_cuda_focuses_the_diffractors(cuda_kernel_factory):
    from pstm_b200 import workloads
    case = workloads.config1()
    k = cuda_kernel_factory(case.config)
    k.migrate_tile(case.traces, case.output, case.velocity)
    for xd, yd, t0 in workloads.C1_DIFFRACTORS:
        xs, ys = neighbourhood(xd, yd)
        check_focus(case.output.image[xs, ys], t0)
