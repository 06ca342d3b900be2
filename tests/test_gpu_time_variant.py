"""Time-variant form on the GPU: the windowed migration is the plain kernel on
the window sample times (bit-identical), the device resampling equals
np.interp, and host and device paths agree."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case():
    from pstm_b200 import workloads
    return workloads.config1(n_traces=1500, nx=10, ny=8, nt=500)


def test_interp_rows_matches_numpy(cuda_kernel_factory):
    import torch
    from pstm_b200 import time_variant as tvm
    rng = np.random.default_rng(0)
    xs = np.cumsum(rng.uniform(0.5, 3.0, 200))
    xd = np.linspace(xs[0] - 5, xs[-1] + 5, 333)
    src = rng.standard_normal((7, 5, 200))
    for dt in (torch.float64, torch.float32):
        got = tvm.interp_rows(torch.as_tensor(src, dtype=dt).cuda(), xs, xd).double().cpu().numpy()
        ref = tvm.interp_rows(src.astype(np.float32 if dt == torch.float32 else np.float64), xs, xd)
        np.testing.assert_allclose(got, ref, rtol=1e-6 if dt == torch.float32 else 1e-13, atol=1e-6)


def test_windowed_migration_is_the_plain_kernel_on_window_times(cuda_kernel_factory):
    from pstm_b200 import time_variant as tvm
    from pstm_b200.base import OutputTile, VelocitySlice
    case = _case()
    k = cuda_kernel_factory(case.config)
    out = case.output
    w = tvm.compute_time_windows(0.0, float(out.t_axis_ms[-1]), 4.0, tvm.FrequencyTimeTable.default())
    tv = tvm.window_times(w)
    assert len(tv) < len(out.t_axis_ms)
    tvo = OutputTile(image=np.zeros(out.image.shape), fold=np.zeros(out.fold.shape, np.int32), x_axis=out.x_axis,
                     y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
    k.migrate_tile_time_variant(case.traces, tvo, case.velocity, case.config, w)
    ref = OutputTile(image=np.zeros(out.image.shape[:2] + (len(tv),)), fold=np.zeros(out.image.shape[:2], np.int32),
                     x_axis=out.x_axis, y_axis=out.y_axis, t_axis_ms=tv)
    k.migrate_tile(case.traces, ref, VelocitySlice(vrms=np.interp(tv, out.t_axis_ms, case.velocity.vrms), is_1d=True))
    np.testing.assert_array_equal(tvo.image, ref.image)
    np.testing.assert_array_equal(tvo.fold, np.broadcast_to(ref.fold[..., None], tvo.fold.shape))
    uni = tvm.resample_to_uniform(tvo.image, w, 4.0, len(out.t_axis_ms))
    assert uni.shape == out.image.shape and np.abs(uni).max() > 0


def test_all_fine_windows_reproduce_migrate_tile_and_device_path(cuda_kernel_factory):
    import torch
    from pstm_b200 import time_variant as tvm
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    case = _case()
    k = cuda_kernel_factory(case.config)
    out = case.output
    fine = tvm.FrequencyTimeTable(times_ms=[0, 5000], frequencies_hz=[400, 300])   # factor 1 everywhere
    w = tvm.compute_time_windows(0.0, float(out.t_axis_ms[-1]) + 4.0, 4.0, fine)
    assert all(x.downsample_factor == 1 for x in w)
    tvo = OutputTile(image=np.zeros(out.image.shape), fold=np.zeros(out.fold.shape, np.int32), x_axis=out.x_axis,
                     y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
    k.migrate_tile_time_variant(case.traces, tvo, case.velocity, case.config, w)
    k.migrate_tile(case.traces, out, case.velocity)
    np.testing.assert_array_equal(tvo.image, out.image)
    np.testing.assert_array_equal(tvo.fold, out.fold)
    # device path: same windows, device tensors
    tb = case.traces
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    w2 = tvm.compute_time_windows(0.0, float(out.t_axis_ms[-1]), 4.0, tvm.FrequencyTimeTable.default())
    host = OutputTile(image=np.zeros(out.image.shape), fold=None, x_axis=out.x_axis, y_axis=out.y_axis,
                      t_axis_ms=out.t_axis_ms)
    k.migrate_tile_time_variant(case.traces, host, case.velocity, case.config, w2)
    do = OutputTile(image=torch.zeros(out.image.shape, dtype=torch.float64, device="cuda"), fold=None,
                    x_axis=dev(out.x_axis), y_axis=dev(out.y_axis), t_axis_ms=dev(out.t_axis_ms))
    k.migrate_tile_time_variant(dtb, do, VelocitySlice(vrms=dev(case.velocity.vrms), is_1d=True), case.config, w2)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(do.image.cpu().numpy(), host.image)
    u_dev = tvm.resample_to_uniform(do.image, w2, 4.0, len(out.t_axis_ms)).cpu().numpy()
    u_host = tvm.resample_to_uniform(host.image, w2, 4.0, len(out.t_axis_ms))
    assert rel_l2(u_dev, u_host) <= 1e-13
