"""The streaming executor: a host-resident panel migrated through a device
pool of midpoint-ordered blocks with the copies overlapped (GPU).

The pool is made tiny (6 slots of 128 traces against 3000 traces) so that
blocks are evicted and reloaded and tiles take several passes; the grid must
equal one resident call with all traces up to the order of the FP32 partial
sums (relative L2 <= 1e-6, fold identical) and the FP64 oracle (<= 1e-5)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["f32", "f16"])
def test_streamed_grid_matches_resident_call_and_oracle(dtype, cuda_kernel_factory):
    import torch
    from oracle import oracle
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.streaming import StreamingExecutor
    sv = workloads.survey(3000, 24, 20, 200, 2.0, 200, seed=3)
    tb = sv.trace_block()
    cfg = workloads.survey_config(aa=True)
    cfg.max_aperture_m = 90.0
    cfg.min_aperture_m = 30.0
    k = cuda_kernel_factory(cfg)
    if dtype == "f16":
        tb = k.to_f16_panel(tb)     # the precision form, host side
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    full, vel = sv.tile(0, 24, 0, 20)
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     weights=None if tb.weights is None else dev(tb.weights),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    ref = OutputTile(image=torch.zeros(full.image.shape, dtype=torch.float64, device="cuda"),
                     fold=torch.zeros(full.fold.shape, dtype=torch.int32, device="cuda"),
                     x_axis=dev(full.x_axis), y_axis=dev(full.y_axis), t_axis_ms=dev(full.t_axis_ms))
    vfull = dev(vel.vrms)
    k.migrate_tile(dtb, ref, VelocitySlice(vrms=vfull, is_1d=False), cfg)
    ex = StreamingExecutor(k, tb, sv.x_axis, sv.y_axis, sv.t_axis_ms,
                           lambda x0, x1, y0, y1: VelocitySlice(vrms=vfull[x0:x1, y0:y1].contiguous(), is_1d=False),
                           cfg, tile=8, block_traces=128, pool_blocks=6)
    img = torch.zeros(full.image.shape, dtype=torch.float64, device="cuda")
    fold = torch.zeros(full.fold.shape, dtype=torch.int32, device="cuda")
    rep = ex.run(img, fold)
    torch.cuda.synchronize()
    assert len(rep.passes) > 9                  # tiles split into several passes
    assert rep.misses > ex.S                    # blocks were evicted and reloaded
    assert rep.h2d_bytes > 0 and rep.kernel_ms > 0
    assert 0.0 <= rep.copy_overlap_ms <= rep.copy_ms + 1e-3 and rep.first_load_ms >= 0.0
    np.testing.assert_array_equal(fold.cpu().numpy(), ref.fold.cpu().numpy())
    assert float(ref.image.abs().max()) > 0
    assert rel_l2(img.cpu().numpy(), ref.image.cpu().numpy()) <= 1e-6
    oref = OutputTile(image=np.zeros(full.image.shape), fold=np.zeros(full.fold.shape, np.int32),
                      x_axis=full.x_axis, y_axis=full.y_axis, t_axis_ms=full.t_axis_ms)
    import dataclasses
    otb = tb
    if dtype == "f16":   # the oracle sees the values the kernel multiplies
        otb = dataclasses.replace(tb, amplitudes=tb.amplitudes.astype(np.float32) *
                                  tb.weights[:, None].astype(np.float32), weights=None)
    oracle.migrate(otb, oref, vel, cfg)
    np.testing.assert_array_equal(fold.cpu().numpy(), oref.fold)
    assert rel_l2(img.cpu().numpy(), oref.image) <= 1e-5
