"""Higher-order trace interpolation (nearest, cubic, windowed sinc, Lanczos)
on the GPU against the FP64 oracle, whose interpolators are pinned to the
reference's interpolate_sample.  On the exact path the kernel works in FP64
like the oracle: relative L2 <= 1e-9, fold bit-exact.  On the fast path (FP64
sample index, FP32 taps, interpolation and weights) the plain bar holds:
relative L2 <= 1e-5."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["exact", "fast"])
@pytest.mark.parametrize("method", ["nearest", "cubic", "sinc4", "sinc8", "sinc16", "lanczos3", "lanczos5"])
def test_interpolators_vs_oracle(method, precision, cuda_kernel_factory):
    import dataclasses
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile
    case = workloads.config1(n_traces=700, nx=6, ny=5, nt=500)
    cfg = dataclasses.replace(case.config, interpolation_method=method, aa_enabled=True)
    k = cuda_kernel_factory(cfg, precision=precision)
    out = case.output
    k.migrate_tile(case.traces, out, case.velocity, cfg)
    ref = OutputTile(image=np.zeros(out.image.shape), fold=np.zeros(out.fold.shape, np.int32), x_axis=out.x_axis,
                     y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
    oracle.migrate(case.traces, ref, case.velocity, cfg)
    np.testing.assert_array_equal(out.fold, ref.fold)
    assert np.abs(ref.image).max() > 0
    assert rel_l2(out.image, ref.image) <= (1e-9 if precision == "exact" else 1e-5)


def test_vti_sinc_and_device_path(cuda_kernel_factory):
    import dataclasses
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    case = workloads.config2_small(n_traces=800, nx=5, ny=4, nt=200, ns=200)
    eta = workloads.survey_eta(case.output.t_axis_ms)
    cfg = workloads.survey_config(kernel_type="anisotropic_vti", aa=True, eta=eta)
    cfg = dataclasses.replace(cfg, interpolation_method="sinc8")
    k = cuda_kernel_factory(cfg)
    out = case.output
    k.migrate_tile_vti(case.traces, out, case.velocity, cfg)
    ref = OutputTile(image=np.zeros(out.image.shape), fold=np.zeros(out.fold.shape, np.int32), x_axis=out.x_axis,
                     y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
    oracle.migrate(case.traces, ref, case.velocity, cfg, kind="anisotropic_vti")
    np.testing.assert_array_equal(out.fold, ref.fold)
    assert rel_l2(out.image, ref.image) <= 1e-9
    tb = case.traces
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    cfg_d = dataclasses.replace(cfg, vti_eta_array=dev(eta))
    d = OutputTile(image=torch.zeros(out.image.shape, dtype=torch.float64, device="cuda"),
                   fold=torch.zeros(out.fold.shape, dtype=torch.int32, device="cuda"),
                   x_axis=dev(out.x_axis), y_axis=dev(out.y_axis), t_axis_ms=dev(out.t_axis_ms))
    k.migrate_tile_vti(dtb, d, VelocitySlice(vrms=dev(case.velocity.vrms), is_1d=False), cfg_d)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.image.cpu().numpy(), out.image)


def test_unknown_method_and_linear_only_forms(cuda_kernel_factory):
    import dataclasses
    from pstm_b200 import workloads
    case = workloads.config1(n_traces=64, nx=4, ny=4, nt=50)
    k = cuda_kernel_factory(case.config)
    with pytest.raises(ValueError, match="interpolation"):
        k.migrate_tile(case.traces, case.output, case.velocity,
                       dataclasses.replace(case.config, interpolation_method="bicubic-ish"))


@pytest.mark.parametrize("method", ["cubic", "sinc8", "lanczos3"])
def test_bf16_traces_rotated_grid_f32_image_2d_fold(method, cuda_kernel_factory):
    """BF16 traces, an FP32 image with a 2-D fold on a rotated grid, a trace count
    that leaves a partial last batch of 128 and an nt that leaves a partial last
    block of 128 times.  The oracle runs on the BF16-rounded samples; the kernel
    accumulates in FP64 and rounds once to FP32 (rel L2 <= 1e-6)."""
    import dataclasses
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile
    from pstm_b200.cuda_kernel import bf16_bits_to_float32, float32_to_bf16_bits
    case = workloads.config1(n_traces=333, nx=5, ny=7, nt=300)
    cfg = dataclasses.replace(case.config, interpolation_method=method, aa_enabled=True)
    out = case.output
    X, Y = np.meshgrid(out.x_axis + 300.0, out.y_axis + 200.0, indexing="ij")
    ang = 0.4
    Xr = 700 + (X - 700) * np.cos(ang) - (Y - 700) * np.sin(ang)
    Yr = 700 + (X - 700) * np.sin(ang) + (Y - 700) * np.cos(ang)
    mk = lambda dt: OutputTile(image=np.zeros(out.image.shape, dt), fold=np.zeros(out.image.shape[:2], np.int32),
                               x_axis=out.x_axis, y_axis=out.y_axis, t_axis_ms=out.t_axis_ms, x_grid=Xr, y_grid=Yr)
    got = mk(np.float32)
    k = cuda_kernel_factory(cfg, trace_dtype="bf16")
    k.migrate_tile(case.traces, got, case.velocity, cfg)
    tb = case.traces
    tq = dataclasses.replace(tb, amplitudes=bf16_bits_to_float32(float32_to_bf16_bits(tb.amplitudes)))
    ref = mk(np.float64)
    oracle.migrate(tq, ref, case.velocity, cfg)
    np.testing.assert_array_equal(got.fold, ref.fold)
    assert ref.fold.max() > 0 and np.abs(ref.image).max() > 0
    assert rel_l2(got.image, ref.image) <= 1e-6
