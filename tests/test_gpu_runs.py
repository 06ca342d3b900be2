"""A tile migrated against row ranges of a resident panel
(pstm_cuda_migrate_tile_runs_dev) vs the same tile migrated against the ranges
gathered into one panel (GPU).  The runs share one tile preparation and one
persistent launch whose items add atomically, so the image equals the gathered
call's up to the FP32 grouping of the partial sums (relative L2 <= 1e-6) and
the fold is identical; a single run takes the per-tile path on the sub-panel
and is bit-identical to it.  The spatial executor (midpoint-ordered panel,
tiles as runs) against one call with all traces closes the loop."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

RUNS = [[0, 0], [10, 700], [900, 2300], [2300, 2301], [3000, 4000]]


def _dev_case(n_traces=4000, kind="straight_ray", **kw):
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import TraceBlock, VelocitySlice
    case = workloads.config2_small(n_traces=n_traces, nx=6, ny=5, nt=300, ns=500)
    eta = workloads.survey_eta(case.output.t_axis_ms) if kind != "straight_ray" else None
    cfg = workloads.survey_config(kernel_type=kind, aa=True, eta=eta)
    cfg = dataclasses.replace(cfg, **kw)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    tb = case.traces
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     weights=dev(np.linspace(0.5, 1.5, n_traces)), sample_rate_ms=tb.sample_rate_ms,
                     start_time_ms=tb.start_time_ms)
    if eta is not None:
        cfg = dataclasses.replace(cfg, vti_eta_array=dev(eta))
    vel = VelocitySlice(vrms=dev(case.velocity.vrms), is_1d=False)
    return case, cfg, dtb, vel, dev


def _out(case, dev, dtype=None):
    import torch
    from pstm_b200.base import OutputTile
    o = case.output
    return OutputTile(image=torch.zeros(o.image.shape, dtype=dtype or torch.float64, device="cuda"),
                      fold=torch.zeros(o.fold.shape, dtype=torch.int32, device="cuda"),
                      x_axis=dev(o.x_axis), y_axis=dev(o.y_axis), t_axis_ms=dev(o.t_axis_ms))


def _gather(tb, idx):
    from pstm_b200.base import TraceBlock
    t = lambda a: a.index_select(0, idx)
    return TraceBlock(amplitudes=t(tb.amplitudes), source_x=t(tb.source_x), source_y=t(tb.source_y),
                      receiver_x=t(tb.receiver_x), receiver_y=t(tb.receiver_y), offset=t(tb.offset),
                      midpoint_x=t(tb.midpoint_x), midpoint_y=t(tb.midpoint_y), weights=t(tb.weights),
                      sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)


@pytest.mark.parametrize("seg_mb", [0, 1])
@pytest.mark.parametrize("kind", ["straight_ray", "anisotropic_vti"])
def test_runs_equal_gathered_panel(kind, seg_mb, cuda_kernel_factory, monkeypatch):
    import torch
    monkeypatch.setenv("PSTM_CUDA_SEGMENT_MB", str(seg_mb))
    case, cfg, dtb, vel, dev = _dev_case(kind=kind)
    k = cuda_kernel_factory(cfg)
    got = _out(case, dev)
    m = k.migrate_tile_runs(dtb, np.array(RUNS), got, vel, cfg, kernel_type=kind)
    idx = torch.as_tensor(np.concatenate([np.arange(a, b) for a, b in RUNS]), device="cuda")
    ref = _out(case, dev)
    (k.migrate_tile if kind == "straight_ray" else k.migrate_tile_vti)(_gather(dtb, idx), ref, vel, cfg)
    torch.cuda.synchronize()
    assert m.n_traces_processed == int(idx.numel())
    np.testing.assert_array_equal(got.fold.cpu().numpy(), ref.fold.cpu().numpy())
    assert float(ref.image.abs().max()) > 0
    assert rel_l2(got.image.cpu().numpy(), ref.image.cpu().numpy()) <= 1e-6
    # the runs against the FP64 oracle on the same traces directly
    from oracle import oracle
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, create_trace_block
    ii = idx.cpu().numpy()
    tb = case.traces
    sub = create_trace_block(tb.amplitudes[ii], tb.source_x[ii], tb.source_y[ii], tb.receiver_x[ii],
                             tb.receiver_y[ii], sample_rate_ms=tb.sample_rate_ms,
                             weights=np.linspace(0.5, 1.5, tb.n_traces)[ii])
    o = case.output
    oref = OutputTile(image=np.zeros(o.image.shape), fold=np.zeros(o.fold.shape, np.int32), x_axis=o.x_axis,
                      y_axis=o.y_axis, t_axis_ms=o.t_axis_ms)
    ocfg = cfg if kind == "straight_ray" else \
        workloads.survey_config(kernel_type=kind, aa=True, eta=workloads.survey_eta(o.t_axis_ms))
    oracle.migrate(sub, oref, case.velocity, ocfg, kind=kind)
    np.testing.assert_array_equal(got.fold.cpu().numpy(), oref.fold)
    assert rel_l2(got.image.cpu().numpy(), oref.image) <= (1e-5 if kind == "straight_ray" else 1e-4)


def test_single_run_no_runs_and_invalid_runs(cuda_kernel_factory):
    import torch
    case, cfg, dtb, vel, dev = _dev_case()
    k = cuda_kernel_factory(cfg)
    got = _out(case, dev, torch.float32)
    k.migrate_tile_runs(dtb, [[0, 0], [1200, 2500], [4000, 4000]], got, vel, cfg)
    idx = torch.arange(1200, 2500, device="cuda")
    ref = _out(case, dev, torch.float32)
    k.migrate_tile(_gather(dtb, idx), ref, vel, cfg)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.image.cpu().numpy(), ref.image.cpu().numpy())
    np.testing.assert_array_equal(got.fold.cpu().numpy(), ref.fold.cpu().numpy())
    before = got.image.clone()
    k.migrate_tile_runs(dtb, np.zeros((0, 2), np.int64), got, vel, cfg)
    k.migrate_tile_runs(dtb, [[5, 5]], got, vel, cfg)
    torch.cuda.synchronize()
    assert torch.equal(got.image, before)
    for bad in ([[10, 20], [15, 30]], [[30, 40], [10, 20]], [[3990, 4001]], [[-1, 5]], [[20, 10]]):
        with pytest.raises(ValueError, match="runs"):
            k.migrate_tile_runs(dtb, bad, got, vel, cfg)
    with pytest.raises(ValueError):
        k.migrate_tile_runs(dtb, [[0, 10]], got, vel, cfg, kernel_type="elliptic")


def test_nonlinear_interpolation_runs(cuda_kernel_factory):
    import torch
    case, cfg, dtb, vel, dev = _dev_case(n_traces=1500, interpolation_method="sinc8")
    k = cuda_kernel_factory(cfg)
    runs = [[0, 400], [700, 1500]]
    got = _out(case, dev)
    k.migrate_tile_runs(dtb, runs, got, vel, cfg)
    idx = torch.as_tensor(np.concatenate([np.arange(a, b) for a, b in runs]), device="cuda")
    ref = _out(case, dev)
    k.migrate_tile(_gather(dtb, idx), ref, vel, cfg)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.fold.cpu().numpy(), ref.fold.cpu().numpy())
    assert rel_l2(got.image.cpu().numpy(), ref.image.cpu().numpy()) <= 1e-12


@pytest.mark.parametrize("spatial", [True, 15.0])
def test_spatial_executor_equals_one_call(spatial, cuda_kernel_factory):
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
    velf = lambda x0, x1, y0, y1: VelocitySlice(vrms=vfull[x0:x1, y0:y1].contiguous(), is_1d=False)
    plain = TiledExecutor(k, dtb, sv.x_axis, sv.y_axis, sv.t_axis_ms, velf, cfg, tile=8)
    ex = TiledExecutor(k, dtb, sv.x_axis, sv.y_axis, sv.t_axis_ms, velf, cfg, tile=8, spatial=spatial)
    img = torch.zeros(full.image.shape, dtype=torch.float64, device="cuda")
    fold = torch.zeros(full.fold.shape, dtype=torch.int32, device="cuda")
    res = ex.run(img, fold)
    torch.cuda.synchronize()
    assert [r.n_traces for r in res] == [int(plain.select(t).numel()) for t in plain.tiles()]
    assert all(r.processed_traces >= r.n_traces for r in res)
    assert sum(r.processed_traces for r in res) < 9 * 3000
    np.testing.assert_array_equal(fold.cpu().numpy(), ref.fold.cpu().numpy())
    assert rel_l2(img.cpu().numpy(), ref.image.cpu().numpy()) <= 1e-6
    sel = ex.select(ex.tiles()[4])
    assert int(sel.numel()) == res[4].n_traces
