"""The trace-centric (scatter) schedule, pstm_cuda_migrate_scatter_dev (GPU).

A midpoint-ordered panel cut into small segments scatters into the whole
grid; the result must equal one gather call with all traces up to the order
of the FP32 partial sums (relative L2 <= 1e-6, fold identical) and the FP64
oracle (straight <= 1e-5, VTI <= 1e-4), and the schedule must hold fewer
items than every segment against every pillar block."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(kind, fold2d=False, seed=3):
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    from pstm_b200.spatial import MidpointIndex, sort_panel
    sv = workloads.survey(3000, 24, 20, 200, 2.0, 200, seed=seed)
    eta = workloads.survey_eta(sv.t_axis_ms) if kind == "anisotropic_vti" else None
    cfg = workloads.survey_config(kernel_type=kind, aa=True, eta=eta)
    cfg.max_aperture_m = 90.0
    cfg.min_aperture_m = 30.0
    tb = sort_panel(sv.trace_block(), MidpointIndex(sv.s[:, 0] * 0.5 + sv.r[:, 0] * 0.5,
                                                    sv.s[:, 1] * 0.5 + sv.r[:, 1] * 0.5, 40.0))
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    full, vel = sv.tile(0, 24, 0, 20)
    fshape = full.image.shape[:2] if fold2d else full.image.shape

    def out():
        return OutputTile(image=torch.zeros(full.image.shape, dtype=torch.float64, device="cuda"),
                          fold=torch.zeros(fshape, dtype=torch.int32, device="cuda"),
                          x_axis=dev(full.x_axis), y_axis=dev(full.y_axis), t_axis_ms=dev(full.t_axis_ms))
    dcfg = cfg
    if eta is not None:
        import dataclasses
        dcfg = dataclasses.replace(cfg, vti_eta_array=dev(eta))
    return tb, dtb, full, vel, VelocitySlice(vrms=dev(vel.vrms), is_1d=False), cfg, dcfg, out, fshape


@pytest.mark.parametrize("kind,fold2d", [("straight_ray", False), ("anisotropic_vti", False),
                                         ("straight_ray", True)])
def test_scatter_equals_gather_and_oracle(kind, fold2d, cuda_kernel_factory):
    import torch
    from oracle import oracle
    from pstm_b200.base import OutputTile
    tb, dtb, full, vel, dvel, cfg, dcfg, out, fshape = _case(kind, fold2d)
    k = cuda_kernel_factory(dcfg)
    got = out()
    m = k.migrate_scatter(dtb, got, dvel, dcfg, kernel_type=kind, segment_traces=64, count_items=True)
    ref = out()
    (k.migrate_tile if kind == "straight_ray" else k.migrate_tile_vti)(dtb, ref, dvel, dcfg)
    torch.cuda.synchronize()
    k.synchronize()
    n_seg = (3000 + 63) // 64   # segments are rounded to whole staged chunks, at least this many traces
    assert 0 < m.n_items < n_seg * (24 * 20)   # far fewer than every segment x every pillar block
    np.testing.assert_array_equal(got.fold.cpu().numpy(), ref.fold.cpu().numpy())
    assert float(ref.image.abs().max()) > 0
    assert rel_l2(got.image.cpu().numpy(), ref.image.cpu().numpy()) <= 1e-6
    oref = OutputTile(image=np.zeros(full.image.shape), fold=np.zeros(fshape, np.int32), x_axis=full.x_axis,
                      y_axis=full.y_axis, t_axis_ms=full.t_axis_ms)
    oracle.migrate(tb, oref, vel, cfg, kind=kind)
    np.testing.assert_array_equal(got.fold.cpu().numpy(), oref.fold)
    assert rel_l2(got.image.cpu().numpy(), oref.image) <= (1e-5 if kind == "straight_ray" else 1e-4)


def test_scatter_rejects_rotated_grids_and_unsorted_axes(cuda_kernel_factory):
    import torch
    from pstm_b200 import _native as nat
    from pstm_b200.base import OutputTile
    tb, dtb, full, vel, dvel, cfg, dcfg, out, fshape = _case("straight_ray")
    k = cuda_kernel_factory(dcfg)
    o = out()
    rot = OutputTile(image=o.image, fold=o.fold, x_axis=o.x_axis, y_axis=o.y_axis, t_axis_ms=o.t_axis_ms,
                     x_grid=torch.zeros(o.image.shape[:2], dtype=torch.float64, device="cuda"),
                     y_grid=torch.zeros(o.image.shape[:2], dtype=torch.float64, device="cuda"))
    with pytest.raises(nat.PstmCudaError) as ei:
        k.migrate_scatter(dtb, rot, dvel, dcfg)
    assert ei.value.code == nat.ERR_UNSUPPORTED
    flipped = OutputTile(image=o.image, fold=o.fold, x_axis=o.x_axis.flip(0).contiguous(), y_axis=o.y_axis,
                         t_axis_ms=o.t_axis_ms)
    k.migrate_scatter(dtb, flipped, dvel, dcfg)   # the check runs on the device
    with pytest.raises(ValueError, match="ascending"):
        k.synchronize()
    o2 = out()   # the context stays usable
    k.migrate_scatter(dtb, o2, dvel, dcfg)
    k.synchronize()
    assert float(o2.image.abs().max()) > 0
