"""The allocation-free entry point, pstm_cuda_migrate_tile_noalloc (GPU).

It serves callers that cannot allocate device memory while they run, so it
keeps its scratch in a fixed array of the library.  The test calls it through
the C ABI with device buffers the test itself allocates, and compares two calls
in a row with the same two calls of the context-based entry point
pstm_cuda_migrate_tile_dev: fold bit-exact, image within the plain-kernel
tolerance (relative L2 <= 1e-5).  After every call it reads the device-side
status back with pstm_cuda_noalloc_status, and one test makes a bounded
wait of the kernel run out (PSTM_CUDA_INJECT_FAULT=wait leaves the first
trace copies unissued) to check that the status reports it.  This file is
collected last on purpose.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _descs(case, dev):
    from pstm_b200 import _native as nat
    tb, out = case.traces, case.output
    keep = {}

    def d(name, a, dtype=np.float64):
        keep[name] = dev(np.ascontiguousarray(a, dtype=dtype))
        return keep[name].data_ptr()

    td = nat.TracesDesc()
    td.amplitudes = d("amps", tb.amplitudes, np.float32)
    td.amp_dtype = nat.AMP_F32
    td.n_samples = tb.n_samples
    td.n_traces = tb.n_traces
    td.amp_row_stride = tb.n_samples
    for f in ("source_x", "source_y", "receiver_x", "receiver_y", "midpoint_x", "midpoint_y"):
        setattr(td, f, d(f, getattr(tb, f)))
    td.sample_rate_ms = tb.sample_rate_ms
    td.start_time_ms = tb.start_time_ms
    vd = nat.VelocityDesc()
    vd.vrms = d("vrms", case.velocity.vrms)
    vd.is_3d = 0
    c = case.config
    pr = nat.Params()
    pr.max_aperture_m, pr.min_aperture_m = c.max_aperture_m, c.min_aperture_m
    pr.max_dip_degrees, pr.taper_fraction = c.max_dip_degrees, c.taper_fraction
    pr.apply_spreading, pr.apply_obliquity = int(c.apply_spreading), int(c.apply_obliquity)
    pr.aa_enabled, pr.traveltime = int(c.aa_enabled), nat.TT_STRAIGHT
    pr.aa_dominant_freq, pr.grid_dx, pr.grid_dy = 30.0, c.grid_dx, c.grid_dy
    pr.curved_v0, pr.curved_k, pr.compensated = 1500.0, 0.5, 1
    axes = (d("x", out.x_axis), d("y", out.y_axis), d("t", out.t_axis_ms))
    return td, vd, pr, axes, keep


def _output(nat, shape, axes, dev_zeros):
    import torch
    img = dev_zeros(shape, torch.float64)
    fold = dev_zeros(shape, torch.int32)
    od = nat.OutputDesc()
    od.image, od.image_dtype, od.fold, od.fold_is_3d = img.data_ptr(), nat.IMAGE_F64, fold.data_ptr(), 1
    od.nx, od.ny, od.nt = shape
    od.x_axis, od.y_axis, od.t_axis_ms = axes
    return od, img, fold


def test_noalloc_matches_context_entry_point_twice():
    import torch
    from pstm_b200 import build, workloads
    from pstm_b200 import _native as nat
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    build.build()
    L = nat.load()
    torch.cuda.set_device(0)
    case = workloads.config1(n_traces=3000, nx=16, ny=12, nt=500)
    dev = lambda a: torch.as_tensor(a, device="cuda")
    zeros = lambda shape, dt: torch.zeros(shape, dtype=dt, device="cuda")
    td, vd, pr, axes, keep = _descs(case, dev)
    shape = case.output.image.shape
    od_ref, img_ref, fold_ref = _output(nat, shape, axes, zeros)
    od_na, img_na, fold_na = _output(nat, shape, axes, zeros)

    ctx = ctypes.c_void_p()
    nat.check(L.pstm_cuda_create(0, ctypes.byref(ctx)), None, L)
    stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY
    try:
        for call in range(2):
            nat.check(L.pstm_cuda_migrate_tile_dev(ctx, ctypes.byref(td), ctypes.byref(od_ref), ctypes.byref(vd),
                                                   ctypes.byref(pr), ctypes.c_void_p(stream)), ctx, L)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            rc = L.pstm_cuda_migrate_tile_noalloc(ctypes.byref(td), ctypes.byref(od_na), ctypes.byref(vd),
                                                  ctypes.byref(pr), ctypes.c_void_p(stream))
            nat.check(rc, None, L)
            nat.check(L.pstm_cuda_noalloc_status(ctypes.c_void_p(stream)), None, L)
            torch.cuda.synchronize()
            if call == 1:   # the first call may load the module; the second must not move memory
                assert torch.cuda.mem_get_info()[0] == free_before
            a, b = img_na.cpu().numpy(), img_ref.cpu().numpy()
            np.testing.assert_array_equal(fold_na.cpu().numpy(), fold_ref.cpu().numpy())
            assert np.linalg.norm(a - b) <= TOL * np.linalg.norm(b)
            assert np.abs(b).max() > 0
    finally:
        L.pstm_cuda_destroy(ctx)


def test_noalloc_rejects_inputs_beyond_its_scratch():
    import torch
    from pstm_b200 import build, workloads
    from pstm_b200 import _native as nat
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    build.build()
    L = nat.load()
    case = workloads.config1(n_traces=64, nx=4, ny=4, nt=50)
    dev = lambda a: torch.as_tensor(a, device="cuda")
    zeros = lambda shape, dt: torch.zeros(shape, dtype=dt, device="cuda")
    td, vd, pr, axes, keep = _descs(case, dev)
    od, img, fold = _output(nat, case.output.image.shape, axes, zeros)
    td.n_traces = 131073   # one more than the fixed scratch holds; nothing is read
    rc = L.pstm_cuda_migrate_tile_noalloc(ctypes.byref(td), ctypes.byref(od), ctypes.byref(vd),
                                          ctypes.byref(pr), None)
    assert rc == nat.ERR_INVALID_ARGUMENT
    assert b"131072" in L.pstm_cuda_last_error(None)
    assert float(img.abs().max()) == 0.0


def test_noalloc_status_reports_a_wait_that_gave_up(monkeypatch):
    """A bounded wait that runs out leaves PSTM_ERR_TIMEOUT in the status; the
    next call clears it and matches the context entry point again."""
    import torch
    from pstm_b200 import build, workloads
    from pstm_b200 import _native as nat
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    build.build()
    L = nat.load()
    torch.cuda.set_device(0)
    case = workloads.config1(n_traces=2000, nx=8, ny=6, nt=500)
    dev = lambda a: torch.as_tensor(a, device="cuda")
    zeros = lambda shape, dt: torch.zeros(shape, dtype=dt, device="cuda")
    td, vd, pr, axes, keep = _descs(case, dev)
    shape = case.output.image.shape
    stream = torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY

    od_bad, img_bad, fold_bad = _output(nat, shape, axes, zeros)
    monkeypatch.setenv("PSTM_CUDA_INJECT_FAULT", "wait")
    rc = L.pstm_cuda_migrate_tile_noalloc(ctypes.byref(td), ctypes.byref(od_bad), ctypes.byref(vd),
                                          ctypes.byref(pr), ctypes.c_void_p(stream))
    assert rc == nat.OK   # asynchronous: the launch itself succeeds
    assert L.pstm_cuda_noalloc_status(ctypes.c_void_p(stream)) == nat.ERR_TIMEOUT
    assert b"partial sums" in L.pstm_cuda_last_error(None)
    monkeypatch.delenv("PSTM_CUDA_INJECT_FAULT")

    od_na, img_na, fold_na = _output(nat, shape, axes, zeros)
    od_ref, img_ref, fold_ref = _output(nat, shape, axes, zeros)
    nat.check(L.pstm_cuda_migrate_tile_noalloc(ctypes.byref(td), ctypes.byref(od_na), ctypes.byref(vd),
                                               ctypes.byref(pr), ctypes.c_void_p(stream)), None, L)
    assert L.pstm_cuda_noalloc_status(ctypes.c_void_p(stream)) == nat.OK
    ctx = ctypes.c_void_p()
    nat.check(L.pstm_cuda_create(0, ctypes.byref(ctx)), None, L)
    try:
        nat.check(L.pstm_cuda_migrate_tile_dev(ctx, ctypes.byref(td), ctypes.byref(od_ref), ctypes.byref(vd),
                                               ctypes.byref(pr), ctypes.c_void_p(stream)), ctx, L)
        torch.cuda.synchronize()
    finally:
        L.pstm_cuda_destroy(ctx)
    a, b = img_na.cpu().numpy(), img_ref.cpu().numpy()
    np.testing.assert_array_equal(fold_na.cpu().numpy(), fold_ref.cpu().numpy())
    assert np.linalg.norm(a - b) <= TOL * np.linalg.norm(b)
