"""Tiled, device-resident migration of a grid vs one call with all traces (GPU).

Traces outside a tile's selection box are outside the aperture of all its
pillars, so the tiled image equals the one-call image up to the FP32 order
of the per-chunk partial sums (relative L2 <= 1e-6) and the fold is identical.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_tiled_grid_equals_one_call(cuda_kernel_factory):
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.executor import TiledExecutor
    sv = workloads.survey(3000, 24, 20, 200, 2.0, 200, seed=3)
    tb = sv.trace_block()
    cfg = workloads.survey_config(aa=True)
    cfg.max_aperture_m = 90.0
    cfg.min_aperture_m = 30.0
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    k = cuda_kernel_factory(cfg)
    full, vel = sv.tile(0, 24, 0, 20)
    ref = OutputTile(image=torch.zeros(full.image.shape, dtype=torch.float64, device="cuda"),
                     fold=torch.zeros(full.fold.shape, dtype=torch.int32, device="cuda"),
                     x_axis=dev(full.x_axis), y_axis=dev(full.y_axis), t_axis_ms=dev(full.t_axis_ms))
    k.migrate_tile(dtb, ref, VelocitySlice(vrms=dev(vel.vrms), is_1d=False), cfg)
    vfull = dev(vel.vrms)
    ex = TiledExecutor(k, dtb, sv.x_axis, sv.y_axis, sv.t_axis_ms,
                       lambda x0, x1, y0, y1: VelocitySlice(vrms=vfull[x0:x1, y0:y1].contiguous(), is_1d=False),
                       cfg, tile=8)
    img = torch.zeros(full.image.shape, dtype=torch.float64, device="cuda")
    fold = torch.zeros(full.fold.shape, dtype=torch.int32, device="cuda")
    res = ex.run(img, fold)
    torch.cuda.synchronize()
    assert len(res) == 9 and sum(r.n_traces for r in res) < 9 * 3000   # the selection prunes
    np.testing.assert_array_equal(fold.cpu().numpy(), ref.fold.cpu().numpy())
    assert rel_l2(img.cpu().numpy(), ref.image.cpu().numpy()) <= 1e-6
    assert float(ref.image.abs().max()) > 0
    # the tiled grid against the FP64 oracle directly: fold bit-exact, image <= 1e-5
    from oracle import oracle
    oref = OutputTile(image=np.zeros(full.image.shape), fold=np.zeros(full.fold.shape, np.int32),
                      x_axis=full.x_axis, y_axis=full.y_axis, t_axis_ms=full.t_axis_ms)
    oracle.migrate(tb, oref, vel, cfg)
    np.testing.assert_array_equal(fold.cpu().numpy(), oref.fold)
    assert rel_l2(img.cpu().numpy(), oref.image) <= 1e-5
