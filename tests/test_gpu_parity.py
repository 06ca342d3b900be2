"""CUDA backend vs the reference's outputs and the FP64 oracle (GPU).

Tolerances (written here, checked below):
* plain straight-ray, FP32 traces (FP64 sample index, the default), vs the
  reference Numba path: fold bit-exact, image relative L2 <= 1e-5;
* the precision form (FP32 traveltime, "fast" with FP64 trace-end re-decisions, "fp32"
  without): <= 1e-3 against the FP64 oracle;
* curved / VTI / curved+VTI / AA / 3-D velocity, FP32 traces, vs the FP64
  oracle: fold bit-exact, image relative L2 <= 1e-5 on the FP64 sample-index
  path ("exact", the default) and <= 1e-4 with FP32 traveltime ("fast");
* BF16 / FP16 traces: <= 1e-5 against the oracle fed the same rounded traces,
  <= 1e-3 against the oracle fed the FP32 traces (FP16 as the precision form
  stores it: one power-of-two scale per trace, carried by the trace weight);
* the precision form on a noise-dominated config-2-shaped tile (1500 samples,
  3-D velocity, AA): FP16 <= 1e-3 against the FP64 oracle on the FP32 traces.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_files, interp_velocity, load_golden_case, rel_l2
from oracle import oracle

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-5
EXACT_KIND_TOL = 1e-5   # every kind on the FP64 sample-index path
FAST_KIND_TOL = 1e-4    # curved / VTI with FP32 traveltime
BF16_TOL = 1e-3


def fresh(out, image_dtype=np.float64, fold_shape=None):
    from pstm_b200.base import OutputTile
    nx, ny, nt = len(out.x_axis), len(out.y_axis), len(out.t_axis_ms)
    return OutputTile(image=np.zeros((nx, ny, nt), image_dtype),
                      fold=np.zeros(fold_shape or (nx, ny, nt), np.int32),
                      x_axis=out.x_axis, y_axis=out.y_axis, t_axis_ms=out.t_axis_ms,
                      x_grid=getattr(out, "x_grid", None), y_grid=getattr(out, "y_grid", None))


def oracle_run(case_traces, out, vel, cfg, kind="straight_ray", pillars=None):
    ref = fresh(out, fold_shape=out.fold.shape)
    oracle.migrate(case_traces, ref, vel, cfg, kind=kind, pillars=pillars)
    return ref


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: os.path.basename(p)[6:-4])
def test_matches_reference_numba_golden(path, cuda_kernel_factory):
    tb, out, vel, cfg, img_ref, fold_ref = load_golden_case(path)
    k = cuda_kernel_factory(cfg)
    k.migrate_tile(tb, out, vel)
    np.testing.assert_array_equal(out.fold, fold_ref)
    if np.abs(img_ref).max() == 0:
        assert np.abs(out.image).max() == 0
    else:
        assert rel_l2(out.image, img_ref) <= PLAIN_TOL


def test_config1_full_tile(cuda_kernel_factory):
    """Full 64x64x500 tile x 16,384 traces; fold everywhere against an FP64
    count, image against the oracle on pillars around the three diffractors."""
    from pstm_b200 import workloads
    case = workloads.config1()
    k = cuda_kernel_factory(case.config)
    k.migrate_tile(case.traces, case.output, case.velocity)
    tb, out = case.traces, case.output
    X, Y = np.meshgrid(out.x_axis, out.y_axis, indexing="ij")
    cnt = np.zeros(X.shape, np.int64)
    for i in range(0, tb.n_traces, 2048):
        d = np.sqrt((X[..., None] - tb.midpoint_x[None, None, i:i + 2048]) ** 2 +
                    (Y[..., None] - tb.midpoint_y[None, None, i:i + 2048]) ** 2)
        cnt += (~(d > case.config.max_aperture_m)).sum(-1)
    np.testing.assert_array_equal(out.fold, np.broadcast_to(cnt[..., None], out.fold.shape))
    ny = out.ny
    for ix in (32, 20, 48):   # rows through (800,800), (500,1100), (1200,400)
        ref = oracle_run(tb, out, case.velocity, case.config, pillars=(ix * ny, (ix + 1) * ny))
        assert rel_l2(out.image[ix], ref.image[ix]) <= PLAIN_TOL


def test_device_tensors_match_host_arrays(cuda_kernel_factory):
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    case = workloads.config1(n_traces=2048, nx=24, ny=20, nt=500)
    k = cuda_kernel_factory(case.config)
    k.migrate_tile(case.traces, case.output, case.velocity)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    tb = case.traces
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    o = case.output
    dout = OutputTile(image=torch.zeros(o.image.shape, dtype=torch.float64, device="cuda"),
                      fold=torch.zeros(o.fold.shape, dtype=torch.int32, device="cuda"),
                      x_axis=dev(o.x_axis), y_axis=dev(o.y_axis), t_axis_ms=dev(o.t_axis_ms))
    k.migrate_tile(dtb, dout, VelocitySlice(vrms=dev(case.velocity.vrms), is_1d=True))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dout.fold.cpu().numpy(), o.fold)
    np.testing.assert_array_equal(dout.image.cpu().numpy(), o.image)


@pytest.mark.parametrize("precision", ["exact", "fast", "fp32"])
@pytest.mark.parametrize("kind", ["straight_ray", "curved_ray", "anisotropic_vti", "curved_vti"])
@pytest.mark.parametrize("aa", [False, True])
def test_traveltime_kinds_vs_oracle(kind, aa, precision, cuda_kernel_factory):
    from pstm_b200 import workloads
    case = workloads.config2_small()
    cfg = workloads.survey_config(kernel_type=kind, aa=aa, eta=workloads.survey_eta(case.output.t_axis_ms),
                                  v0=1500.0, k=0.9)
    k = cuda_kernel_factory(cfg, precision=precision)
    method = {"straight_ray": k.migrate_tile, "curved_ray": k.migrate_tile_curved_ray,
              "anisotropic_vti": k.migrate_tile_vti, "curved_vti": k.migrate_tile_curved_vti}[kind]
    method(case.traces, case.output, case.velocity)
    ref = oracle_run(case.traces, case.output, case.velocity, cfg, kind=kind)
    np.testing.assert_array_equal(case.output.fold, ref.fold)
    err = rel_l2(case.output.image, ref.image)
    tol = EXACT_KIND_TOL if (precision == "exact" or kind == "straight_ray") else FAST_KIND_TOL
    assert err <= tol, err


@pytest.mark.parametrize("precision", ["exact", "fast", "fp32"])
def test_curved_zero_gradient_and_constant_eta(precision, cuda_kernel_factory):
    from pstm_b200 import workloads
    case = workloads.config2_small(n_traces=1024, nx=8, ny=8)
    cfg = workloads.survey_config(kernel_type="curved_ray", aa=False, v0=1700.0, k=0.0)
    k = cuda_kernel_factory(cfg, precision=precision)
    tol = EXACT_KIND_TOL if precision == "exact" else FAST_KIND_TOL
    k.migrate_tile_curved_ray(case.traces, case.output, case.velocity)
    ref = oracle_run(case.traces, case.output, case.velocity, cfg, kind="curved_ray")
    assert rel_l2(case.output.image, ref.image) <= tol
    cfg2 = workloads.survey_config(kernel_type="anisotropic_vti", aa=False)
    cfg2.vti_eta_array = None
    cfg2.vti_eta_constant = 0.12
    out = fresh(case.output)
    k.migrate_tile_vti(case.traces, out, case.velocity, cfg2)
    ref = oracle_run(case.traces, out, case.velocity, cfg2, kind="anisotropic_vti")
    assert rel_l2(out.image, ref.image) <= tol
    # curved + VTI with a zero gradient: straight legs in v0, the VTI ratio in v_rms
    cfg3 = workloads.survey_config(kernel_type="curved_vti", aa=True, v0=1700.0, k=0.0,
                                   eta=workloads.survey_eta(case.output.t_axis_ms))
    out3 = fresh(case.output)
    k.migrate_tile_curved_vti(case.traces, out3, case.velocity, cfg3)
    ref3 = oracle_run(case.traces, out3, case.velocity, cfg3, kind="curved_vti")
    assert rel_l2(out3.image, ref3.image) <= tol


@pytest.mark.parametrize("precision", ["exact", "fast", "fp32"])
@pytest.mark.parametrize("dtype", ["bf16", "f16"])
def test_16bit_traces(dtype, precision, cuda_kernel_factory):
    from pstm_b200 import workloads
    from pstm_b200.cuda_kernel import bf16_bits_to_float32, float32_to_bf16_bits
    case = workloads.config2_small()
    k = cuda_kernel_factory(case.config, trace_dtype=dtype, precision=precision)
    k.migrate_tile(case.traces, case.output, case.velocity)
    tb = case.traces
    if dtype == "bf16":
        q = bf16_bits_to_float32(float32_to_bf16_bits(tb.amplitudes))
    else:   # the values the kernel multiplies: scaled FP16 times the trace's inverse scale
        from pstm_b200.cuda_kernel import scaled_f16
        a16, inv = scaled_f16(tb.amplitudes)
        q = a16.astype(np.float32) * inv[:, None].astype(np.float32)
    import dataclasses
    tq = dataclasses.replace(tb, amplitudes=q)
    ref_q = oracle_run(tq, case.output, case.velocity, case.config)
    ref = oracle_run(tb, case.output, case.velocity, case.config)
    np.testing.assert_array_equal(case.output.fold, ref.fold)
    if precision == "exact":
        assert rel_l2(case.output.image, ref_q.image) <= PLAIN_TOL
    assert rel_l2(case.output.image, ref.image) <= BF16_TOL


def _noise_tile(n_traces=16384, pillars=8, seed=3):
    """A config-2-shaped tile whose panel is pure Gaussian noise (the case
    where trace quantisation shows most): 1500 samples at 2 ms, 3.2 km patch,
    3-D v_rms, AA on, 8 x 8 pillars at the grid centre x 1500 output times."""
    from pstm_b200 import workloads
    sv = workloads.survey(n_traces, 256, 256, 1500, 2.0, 1500, seed=seed, with_amplitudes=False)
    rng = np.random.default_rng(seed)
    amps = rng.standard_normal((n_traces, 1500)).astype(np.float32) * \
        rng.uniform(0.01, 100.0, n_traces).astype(np.float32)[:, None]   # uneven trace levels
    sv.amps = amps
    c0 = 128 - pillars // 2
    out, vel = sv.tile(c0, c0 + pillars, c0, c0 + pillars)
    return sv.trace_block(), out, vel, workloads.survey_config(aa=True)


@pytest.mark.parametrize("precision", ["exact", "fast", "fp32"])
def test_precision_form_noise_dominated_config2_tile(precision, cuda_kernel_factory):
    from pstm_b200.cuda_kernel import bf16_bits_to_float32, float32_to_bf16_bits
    tb, out, vel, cfg = _noise_tile()
    ref = oracle_run(tb, out, vel, cfg)
    k16 = cuda_kernel_factory(cfg, trace_dtype="f16", precision=precision)
    o16 = fresh(out)
    k16.migrate_tile(tb, o16, vel)
    np.testing.assert_array_equal(o16.fold, ref.fold)
    err16 = rel_l2(o16.image, ref.image)
    assert err16 <= BF16_TOL, err16
    # why the form is FP16: BF16 keeps 8 significant bits, and its rounding of a
    # noise panel alone is above the bar (checked on the rounded traces, CPU)
    import dataclasses
    tq = dataclasses.replace(tb, amplitudes=bf16_bits_to_float32(float32_to_bf16_bits(tb.amplitudes)))
    ref_bf = oracle_run(tq, out, vel, cfg, pillars=(0, 16))   # pillars ix 0-1, all iy
    assert rel_l2(ref_bf.image[:2], ref.image[:2]) > BF16_TOL


def test_f16_panel_device_matches_host_rule(cuda_kernel_factory):
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import TraceBlock
    from pstm_b200.cuda_kernel import scaled_f16
    case = workloads.config1(n_traces=3000, nx=4, ny=4, nt=50)
    tb = case.traces
    a = tb.amplitudes.copy()
    a[5] = 0.0                       # an all-zero trace keeps scale 1
    a[7] *= 1e-9                     # tiny and large levels both land in [2^13, 2^14)
    a[9] *= 1e9
    k = cuda_kernel_factory(case.config)
    dev = lambda x: torch.as_tensor(np.ascontiguousarray(x), device="cuda")
    w = np.linspace(0.5, 2.0, a.shape[0])
    dtb = TraceBlock(amplitudes=dev(a), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y), weights=dev(w),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    d16 = k.to_f16_panel(dtb)
    h16, inv = scaled_f16(a)
    np.testing.assert_array_equal(d16.amplitudes.cpu().numpy().view(np.uint16), h16.view(np.uint16))
    np.testing.assert_array_equal(d16.weights.cpu().numpy(), w * inv)


@pytest.mark.parametrize("precision", ["fast", "fp32"])
@pytest.mark.parametrize("path", golden_files(), ids=lambda p: os.path.basename(p)[6:-4])
def test_fast_precision_form_on_golden(path, precision, cuda_kernel_factory):
    """FP32 traveltime (with and without the FP64 trace-end re-decisions)
    against the reference outputs."""
    tb, out, vel, cfg, img_ref, fold_ref = load_golden_case(path)
    k = cuda_kernel_factory(cfg, precision=precision)
    k.migrate_tile(tb, out, vel)
    np.testing.assert_array_equal(out.fold, fold_ref)
    if np.abs(img_ref).max() > 0:
        assert rel_l2(out.image, img_ref) <= BF16_TOL


def test_edge_shapes_rotated_grid_f32_image_2d_fold(cuda_kernel_factory):
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile
    case = workloads.config1(n_traces=700, nx=7, ny=13, nt=37)
    c = case.config
    out = case.output
    X, Y = np.meshgrid(out.x_axis + 300.0, out.y_axis + 200.0, indexing="ij")
    ang = 0.3
    Xr = 700 + (X - 700) * np.cos(ang) - (Y - 700) * np.sin(ang)
    Yr = 700 + (X - 700) * np.sin(ang) + (Y - 700) * np.cos(ang)
    rot = OutputTile(image=np.zeros(out.image.shape, np.float32), fold=np.zeros(out.image.shape[:2], np.int32),
                     x_axis=out.x_axis, y_axis=out.y_axis, t_axis_ms=out.t_axis_ms, x_grid=Xr, y_grid=Yr)
    k = cuda_kernel_factory(c)
    k.migrate_tile(case.traces, rot, case.velocity)
    ref = oracle_run(case.traces, rot, case.velocity, c)
    np.testing.assert_array_equal(rot.fold, ref.fold)
    assert rel_l2(rot.image, ref.image) <= PLAIN_TOL


def test_zero_and_single_trace(cuda_kernel_factory):
    from pstm_b200 import workloads
    from pstm_b200.base import create_trace_block
    case = workloads.config1(n_traces=1, nx=5, ny=5, nt=40)
    k = cuda_kernel_factory(case.config)
    k.migrate_tile(case.traces, case.output, case.velocity)
    ref = oracle_run(case.traces, case.output, case.velocity, case.config)
    np.testing.assert_array_equal(case.output.fold, ref.fold)
    assert rel_l2(case.output.image, ref.image) <= PLAIN_TOL
    empty = create_trace_block(np.zeros((0, 500), np.float32), *([np.zeros(0)] * 4), sample_rate_ms=4.0)
    before_i, before_f = case.output.image.copy(), case.output.fold.copy()
    k.migrate_tile(empty, case.output, case.velocity)
    np.testing.assert_array_equal(case.output.image, before_i)
    np.testing.assert_array_equal(case.output.fold, before_f)


def test_additive_over_trace_splits_and_exact_scaling(cuda_kernel_factory):
    """Size-independent properties: fold and image add over a split of the
    traces; scaling the traces by 2 scales the image by exactly 2."""
    import dataclasses
    from pstm_b200 import workloads
    case = workloads.config1(n_traces=6000, nx=16, ny=16, nt=500)
    k = cuda_kernel_factory(case.config)
    tb = case.traces
    k.migrate_tile(tb, case.output, case.velocity)
    split = fresh(case.output)
    half = tb.n_traces // 2
    for sl in (slice(0, half), slice(half, None)):
        part = dataclasses.replace(tb, **{f: getattr(tb, f)[sl] for f in
                                          ("amplitudes", "source_x", "source_y", "receiver_x", "receiver_y",
                                           "offset", "midpoint_x", "midpoint_y")})
        k.migrate_tile(part, split, case.velocity)
    np.testing.assert_array_equal(split.fold, case.output.fold)
    assert rel_l2(split.image, case.output.image) <= 1e-6
    doubled = fresh(case.output)
    k.migrate_tile(dataclasses.replace(tb, amplitudes=tb.amplitudes * 2), doubled, case.velocity)
    np.testing.assert_allclose(doubled.image, 2 * case.output.image, rtol=1e-6, atol=0)


def test_invalid_arguments_and_injected_fault(cuda_kernel_factory, monkeypatch):
    from pstm_b200 import workloads
    from pstm_b200._native import PstmCudaError
    case = workloads.config1(n_traces=64, nx=4, ny=4, nt=20)
    k = cuda_kernel_factory(case.config)
    bad = workloads.config1(n_traces=64, nx=4, ny=4, nt=20)
    bad.velocity.vrms[:] = 0.0
    with pytest.raises(ValueError):
        k.migrate_tile(bad.traces, bad.output, bad.velocity)
    monkeypatch.setenv("PSTM_CUDA_INJECT_FAULT", "migrate")
    with pytest.raises(PstmCudaError, match="INJECTED"):
        k.migrate_tile(case.traces, case.output, case.velocity)
    monkeypatch.delenv("PSTM_CUDA_INJECT_FAULT")
    k.migrate_tile(case.traces, case.output, case.velocity)   # context still usable
    ref = oracle_run(case.traces, case.output, case.velocity, case.config)
    assert rel_l2(case.output.image, ref.image) <= PLAIN_TOL


def test_compensated_partials(cuda_kernel_factory):
    """TwoSum-compensated partial sums (the precision form's accumulation) stay
    within the plain tolerance and no farther from the FP64 oracle than the
    plain FP32 partials."""
    from pstm_b200 import workloads
    case = workloads.config1(n_traces=4000, nx=8, ny=6, nt=500)
    out = case.output
    ref = oracle_run(case.traces, out, case.velocity, case.config)
    errs = {}
    for comp in (False, True):
        k = cuda_kernel_factory(case.config, compensated=comp)
        o = fresh(out)
        k.migrate_tile(case.traces, o, case.velocity)
        np.testing.assert_array_equal(o.fold, ref.fold)
        errs[comp] = rel_l2(o.image, ref.image)
    assert errs[True] <= PLAIN_TOL and errs[True] <= errs[False] * 1.05 + 1e-9, errs
