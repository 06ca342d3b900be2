"""The batched form: many offset bins of one tile in one persistent launch,
replayed from a CUDA graph, with the autotuner (GPU).

Each bin of the batch must equal what the per-tile entry point gives for that
bin's traces alone: with the default launch shape the two run the same
arithmetic in the same order, so image and fold are compared bit for bit; a
tuned shape changes the FP32 partial-sum order, so it is held to the plain
tolerance (relative L2 <= 1e-5) against the per-tile result, and one bin is
checked against the FP64 oracle at the kind's tolerance.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-5
KIND_TOL = 1e-4


def _batch(counts, nx=12, ny=10, nt=300, ns=300, seed=11, kind="straight_ray"):
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    bs = workloads.binned_survey(counts, nx, ny, nt, 2.0, ns, seed=seed)
    sv = bs.survey
    tb = sv.trace_block()
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    out, vel = sv.tile(0, nx, 0, ny)
    geo = OutputTile(image=None, fold=None, x_axis=dev(out.x_axis), y_axis=dev(out.y_axis),
                     t_axis_ms=dev(out.t_axis_ms))
    dvel = VelocitySlice(vrms=dev(vel.vrms), is_1d=False)
    eta = workloads.survey_eta(out.t_axis_ms) if kind in ("anisotropic_vti", "curved_vti") else None
    cfg = workloads.survey_config(kernel_type=kind, aa=True, eta=eta)
    if eta is not None:
        cfg.vti_eta_array = dev(eta)
    return bs, tb, dtb, out, vel, geo, dvel, cfg


def _outputs(n, shape, fold3=True):
    import torch
    imgs = [torch.zeros(shape, dtype=torch.float64, device="cuda") for _ in range(n)]
    folds = [torch.zeros(shape if fold3 else shape[:2], dtype=torch.int32, device="cuda") for _ in range(n)]
    return imgs, folds


def _per_tile(k, dtb, geo, dvel, cfg, kind, b0, n, shape, calls=1):
    """One bin through the per-tile device entry point."""
    import torch
    from pstm_b200.base import OutputTile, TraceBlock
    sl = slice(int(b0), int(b0 + n))
    sub = TraceBlock(amplitudes=dtb.amplitudes[sl], source_x=dtb.source_x[sl], source_y=dtb.source_y[sl],
                     receiver_x=dtb.receiver_x[sl], receiver_y=dtb.receiver_y[sl], offset=dtb.offset[sl],
                     midpoint_x=dtb.midpoint_x[sl], midpoint_y=dtb.midpoint_y[sl],
                     sample_rate_ms=dtb.sample_rate_ms, start_time_ms=dtb.start_time_ms)
    o = OutputTile(image=torch.zeros(shape, dtype=torch.float64, device="cuda"),
                   fold=torch.zeros(shape, dtype=torch.int32, device="cuda"),
                   x_axis=geo.x_axis, y_axis=geo.y_axis, t_axis_ms=geo.t_axis_ms)
    method = {"straight_ray": k.migrate_tile, "curved_ray": k.migrate_tile_curved_ray,
              "anisotropic_vti": k.migrate_tile_vti, "curved_vti": k.migrate_tile_curved_vti}[kind]
    for _ in range(calls):
        if n > 0:
            method(sub, o, dvel, cfg)
    torch.cuda.synchronize()
    return o.image.cpu().numpy(), o.fold.cpu().numpy()


@pytest.mark.parametrize("kind", ["straight_ray", "anisotropic_vti", "curved_vti"])
def test_bins_match_per_tile_calls_bitwise(kind, cuda_kernel_factory):
    import torch
    from pstm_b200.cuda_kernel import Bin
    counts = [700, 0, 2500, 40, 1300]   # uneven, one empty bin
    bs, tb, dtb, out, vel, geo, dvel, cfg = _batch(counts, kind=kind)
    k = cuda_kernel_factory(cfg)
    shape = out.image.shape
    imgs, folds = _outputs(len(counts), shape)
    bins = [Bin(b0, n, imgs[i], folds[i]) for i, (b0, n) in enumerate(zip(bs.starts, bs.counts))]
    k.migrate_bins(dtb, bins, geo, dvel, cfg, kernel_type=kind)
    torch.cuda.synchronize()
    k.synchronize()
    for i, (b0, n) in enumerate(zip(bs.starts, bs.counts)):
        ref_img, ref_fold = _per_tile(k, dtb, geo, dvel, cfg, kind, b0, n, shape)
        np.testing.assert_array_equal(folds[i].cpu().numpy(), ref_fold)
        np.testing.assert_array_equal(imgs[i].cpu().numpy(), ref_img)
    assert float(imgs[1].abs().max()) == 0.0 and int(folds[1].abs().max()) == 0   # the empty bin
    # one bin against the FP64 oracle
    from pstm_b200.base import OutputTile, create_trace_block
    i = 2
    sl = slice(int(bs.starts[i]), int(bs.starts[i] + bs.counts[i]))
    sub = create_trace_block(tb.amplitudes[sl], tb.source_x[sl], tb.source_y[sl], tb.receiver_x[sl],
                             tb.receiver_y[sl], sample_rate_ms=tb.sample_rate_ms)
    ref = OutputTile(image=np.zeros(shape), fold=np.zeros(shape, np.int32), x_axis=out.x_axis,
                     y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
    ocfg = cfg
    if kind != "straight_ray":
        from pstm_b200 import workloads
        ocfg = workloads.survey_config(kernel_type=kind, aa=True, eta=workloads.survey_eta(out.t_axis_ms))
    oracle.migrate(sub, ref, vel, ocfg, kind=kind)
    np.testing.assert_array_equal(folds[i].cpu().numpy(), ref.fold)
    tol = PLAIN_TOL if kind == "straight_ray" else KIND_TOL
    assert rel_l2(imgs[i].cpu().numpy(), ref.image) <= tol


def test_graph_replay_recapture_and_direct_launch(cuda_kernel_factory, monkeypatch):
    """Two calls with the same arguments replay the captured graph (image and
    fold accumulate twice, exactly as two per-tile calls); new bins re-capture;
    PSTM_CUDA_GRAPH=0 launches without a graph and gives the same bits."""
    import torch
    from pstm_b200.cuda_kernel import Bin
    counts = [900, 300, 1600]
    bs, tb, dtb, out, vel, geo, dvel, cfg = _batch(counts, seed=21)
    k = cuda_kernel_factory(cfg)
    shape = out.image.shape
    imgs, folds = _outputs(3, shape)
    bins = [Bin(b0, n, imgs[i], folds[i]) for i, (b0, n) in enumerate(zip(bs.starts, bs.counts))]
    for _ in range(2):
        k.migrate_bins(dtb, bins, geo, dvel, cfg)
    torch.cuda.synchronize()
    k.synchronize()
    refs = [_per_tile(k, dtb, geo, dvel, cfg, "straight_ray", b0, n, shape, calls=2)
            for b0, n in zip(bs.starts, bs.counts)]
    for i in range(3):
        np.testing.assert_array_equal(imgs[i].cpu().numpy(), refs[i][0])
        np.testing.assert_array_equal(folds[i].cpu().numpy(), refs[i][1])

    # other bins (the last two swapped and split differently): a new capture
    imgs2, folds2 = _outputs(2, shape)
    split = [(0, 1200), (1200, 1600)]
    bins2 = [Bin(b0, n, imgs2[i], folds2[i]) for i, (b0, n) in enumerate(split)]
    k.migrate_bins(dtb, bins2, geo, dvel, cfg)
    torch.cuda.synchronize()
    for i, (b0, n) in enumerate(split):
        ref_img, ref_fold = _per_tile(k, dtb, geo, dvel, cfg, "straight_ray", b0, n, shape)
        np.testing.assert_array_equal(imgs2[i].cpu().numpy(), ref_img)
        np.testing.assert_array_equal(folds2[i].cpu().numpy(), ref_fold)

    monkeypatch.setenv("PSTM_CUDA_GRAPH", "0")
    imgs3, folds3 = _outputs(2, shape)
    bins3 = [Bin(b0, n, imgs3[i], folds3[i]) for i, (b0, n) in enumerate(split)]
    k.migrate_bins(dtb, bins3, geo, dvel, cfg)
    torch.cuda.synchronize()
    for i in range(2):
        np.testing.assert_array_equal(imgs3[i].cpu().numpy(), imgs2[i].cpu().numpy())
        np.testing.assert_array_equal(folds3[i].cpu().numpy(), folds2[i].cpu().numpy())


def test_autotune_then_batch(cuda_kernel_factory):
    import torch
    from pstm_b200.cuda_kernel import Bin
    counts = [3000, 500, 1800, 60]
    bs, tb, dtb, out, vel, geo, dvel, cfg = _batch(counts, nx=24, ny=20, nt=600, ns=600, seed=31,
                                                   kind="anisotropic_vti")
    k = cuda_kernel_factory(cfg)
    shape = out.image.shape
    imgs, folds = _outputs(len(counts), shape)
    bins = [Bin(b0, n, imgs[i], folds[i]) for i, (b0, n) in enumerate(zip(bs.starts, bs.counts))]
    res = k.autotune_bins(dtb, bins, geo, dvel, cfg, kernel_type="anisotropic_vti", pairs_per_candidate=1 << 30)
    assert res["n_candidates"] >= 2
    assert 0 < res["best_ms"] <= res["default_ms"]
    assert 1 <= res["pillars_per_cta"] <= 16 and 1 <= res["times_per_lane"] <= 8
    assert float(sum(float(i.abs().max()) for i in imgs)) == 0.0   # tuning writes only its own scratch
    k.migrate_bins(dtb, bins, geo, dvel, cfg, kernel_type="anisotropic_vti")
    torch.cuda.synchronize()
    k.synchronize()
    for i, (b0, n) in enumerate(zip(bs.starts, bs.counts)):
        ref_img, ref_fold = _per_tile(k, dtb, geo, dvel, cfg, "anisotropic_vti", b0, n, shape)
        np.testing.assert_array_equal(folds[i].cpu().numpy(), ref_fold)
        assert rel_l2(imgs[i].cpu().numpy(), ref_img) <= PLAIN_TOL


def test_batch_argument_checks(cuda_kernel_factory):
    import torch
    from pstm_b200.cuda_kernel import Bin
    bs, tb, dtb, out, vel, geo, dvel, cfg = _batch([200, 100], nx=6, ny=5, nt=100, ns=100)
    k = cuda_kernel_factory(cfg)
    shape = out.image.shape
    imgs, folds = _outputs(2, shape)
    with pytest.raises(ValueError, match="overlap"):
        k.migrate_bins(dtb, [Bin(0, 200, imgs[0]), Bin(200, 100, imgs[0])], geo, dvel, cfg)
    with pytest.raises(ValueError, match="outside"):
        k.migrate_bins(dtb, [Bin(250, 100, imgs[0])], geo, dvel, cfg)
    with pytest.raises(ValueError, match="CUDA"):
        k.migrate_bins(dtb, [Bin(0, 200, np.zeros(shape))], geo, dvel, cfg)
    k.migrate_bins(dtb, [], geo, dvel, cfg)   # nothing to do
    k.migrate_bins(dtb, [Bin(0, 0, imgs[1], folds[1])], geo, dvel, cfg)   # an empty bin
    torch.cuda.synchronize()
    assert float(imgs[0].abs().max()) == 0.0 and float(imgs[1].abs().max()) == 0.0


def test_bins_split_into_trace_segments(cuda_kernel_factory, monkeypatch):
    """With 1 MiB segments the larger bins are split into trace segments that
    add into their outputs atomically: same fold, image within 1e-6 of the
    unsplit per-tile result."""
    import torch
    from pstm_b200.cuda_kernel import Bin
    counts = [2500, 300, 1800]
    bs, tb, dtb, out, vel, geo, dvel, cfg = _batch(counts, seed=41)
    monkeypatch.setenv("PSTM_CUDA_SEGMENT_MB", "1")
    k = cuda_kernel_factory(cfg)
    monkeypatch.setenv("PSTM_CUDA_SEGMENT_MB", "0")
    k_ref = cuda_kernel_factory(cfg)
    shape = out.image.shape
    imgs, folds = _outputs(len(counts), shape)
    bins = [Bin(b0, n, imgs[i], folds[i]) for i, (b0, n) in enumerate(zip(bs.starts, bs.counts))]
    k.migrate_bins(dtb, bins, geo, dvel, cfg)
    torch.cuda.synchronize()
    k.synchronize()
    for i, (b0, n) in enumerate(zip(bs.starts, bs.counts)):
        ref_img, ref_fold = _per_tile(k_ref, dtb, geo, dvel, cfg, "straight_ray", b0, n, shape)
        np.testing.assert_array_equal(folds[i].cpu().numpy(), ref_fold)
        assert rel_l2(imgs[i].cpu().numpy(), ref_img) <= 1e-6


@pytest.mark.parametrize("kind", ["straight_ray", "anisotropic_vti"])
def test_autotuned_segmented_batch_vs_fp64_oracle(kind, cuda_kernel_factory, monkeypatch):
    """The whole composite path -- autotuned launch shape, bins split into
    1 MiB trace segments with atomic adds, one graph-replayed persistent
    launch -- against the FP64 oracle bin by bin: fold bit-exact, image within
    the kind's tolerance."""
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, create_trace_block
    from pstm_b200.cuda_kernel import Bin
    counts = [2600, 400, 1900, 30]
    bs, tb, dtb, out, vel, geo, dvel, cfg = _batch(counts, nx=20, ny=16, nt=400, ns=400, seed=51, kind=kind)
    monkeypatch.setenv("PSTM_CUDA_SEGMENT_MB", "1")
    k = cuda_kernel_factory(cfg)
    shape = out.image.shape
    imgs, folds = _outputs(len(counts), shape)
    bins = [Bin(b0, n, imgs[i], folds[i]) for i, (b0, n) in enumerate(zip(bs.starts, bs.counts))]
    k.autotune_bins(dtb, bins, geo, dvel, cfg, kernel_type=kind, pairs_per_candidate=1 << 29)
    k.migrate_bins(dtb, bins, geo, dvel, cfg, kernel_type=kind)
    torch.cuda.synchronize()
    k.synchronize()
    ocfg = cfg if kind == "straight_ray" else \
        workloads.survey_config(kernel_type=kind, aa=True, eta=workloads.survey_eta(out.t_axis_ms))
    tol = PLAIN_TOL if kind == "straight_ray" else KIND_TOL
    for i, (b0, n) in enumerate(zip(bs.starts, bs.counts)):
        sl = slice(int(b0), int(b0 + n))
        sub = create_trace_block(tb.amplitudes[sl], tb.source_x[sl], tb.source_y[sl], tb.receiver_x[sl],
                                 tb.receiver_y[sl], sample_rate_ms=tb.sample_rate_ms)
        ref = OutputTile(image=np.zeros(shape), fold=np.zeros(shape, np.int32), x_axis=out.x_axis,
                         y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
        oracle.migrate(sub, ref, vel, ocfg, kind=kind)
        np.testing.assert_array_equal(folds[i].cpu().numpy(), ref.fold)
        assert rel_l2(imgs[i].cpu().numpy(), ref.image) <= tol, (i, kind)
