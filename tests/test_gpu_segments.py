"""Large panels run segment by segment through the persistent kernel with
atomic image/fold adds (GPU).  Forced here on a small panel with 1 MiB
segments: the result equals the unsegmented launch up to the FP32 grouping
of the partial sums (relative L2 <= 1e-6), the fold is identical, and both
match the FP64 oracle to the plain tolerance (1e-5)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["straight_ray", "anisotropic_vti"])
def test_segmented_equals_unsegmented(kind, cuda_kernel_factory, monkeypatch):
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile
    case = workloads.config2_small(n_traces=3000, nx=6, ny=5, nt=300, ns=500)
    eta = workloads.survey_eta(case.output.t_axis_ms) if kind != "straight_ray" else None
    cfg = workloads.survey_config(kernel_type=kind, aa=True, eta=eta)
    out = case.output

    def run(seg_mb):
        monkeypatch.setenv("PSTM_CUDA_SEGMENT_MB", str(seg_mb))
        k = cuda_kernel_factory(cfg)
        o = OutputTile(image=np.zeros(out.image.shape), fold=np.zeros(out.fold.shape, np.int32),
                       x_axis=out.x_axis, y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
        (k.migrate_tile if kind == "straight_ray" else k.migrate_tile_vti)(case.traces, o, case.velocity, cfg)
        return o

    seg, whole = run(1), run(0)
    np.testing.assert_array_equal(seg.fold, whole.fold)
    assert rel_l2(seg.image, whole.image) <= 1e-6
    ref = OutputTile(image=np.zeros(out.image.shape), fold=np.zeros(out.fold.shape, np.int32),
                     x_axis=out.x_axis, y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
    oracle.migrate(case.traces, ref, case.velocity, cfg, kind=kind)
    np.testing.assert_array_equal(seg.fold, ref.fold)
    assert rel_l2(seg.image, ref.image) <= (1e-5 if kind == "straight_ray" else 1e-4)
