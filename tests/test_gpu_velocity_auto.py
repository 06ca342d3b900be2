"""``CudaKernel(velocity_mode="auto")`` on the GPU: with small lateral variation
the tile is migrated with the centre pillar (bit-identical to passing that
1-D velocity), with large variation with the cube (bit-identical to the exact
mode); host arrays and CUDA tensors alike (metal_compiled.py:631-664)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("on_device", [False, True])
@pytest.mark.parametrize("scale,is3d", [(0.1, False), (3.0, True)])
def test_auto_velocity(scale, is3d, on_device, cuda_kernel_factory):
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, VelocitySlice
    case = workloads.config2_small(n_traces=500, nx=6, ny=5, nt=100, ns=200)
    v = np.asarray(case.velocity.vrms, np.float64)
    centre = v[3, 2, :]
    v3 = centre[None, None, :] + scale * (v - centre[None, None, :])
    rel = np.abs(v3 - centre[None, None, :]).max() / centre.mean()
    assert (rel > 0.05) == is3d
    o = case.output
    dev = (lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()) if on_device else (lambda a: a)
    tb = case.traces
    if on_device:
        from pstm_b200.base import TraceBlock
        tb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                        receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                        midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                        sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)

    def run(kernel, vel):
        out = OutputTile(image=dev(np.zeros(o.image.shape)), fold=dev(np.zeros(o.fold.shape, np.int32)),
                         x_axis=dev(o.x_axis), y_axis=dev(o.y_axis), t_axis_ms=dev(o.t_axis_ms))
        kernel.migrate_tile(tb, out, vel, case.config)
        torch.cuda.synchronize()
        return np.asarray(out.image.cpu() if on_device else out.image)

    auto = run(cuda_kernel_factory(case.config, velocity_mode="auto"), VelocitySlice(vrms=dev(v3), is_1d=False))
    plain = cuda_kernel_factory(case.config)
    want = run(plain, VelocitySlice(vrms=dev(v3), is_1d=False)) if is3d else \
        run(plain, VelocitySlice(vrms=dev(np.ascontiguousarray(centre)), is_1d=True))
    assert np.abs(want).max() > 0
    np.testing.assert_array_equal(auto, want)
