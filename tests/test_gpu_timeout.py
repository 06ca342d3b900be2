"""Device-side failure detection of the context entry points (GPU).

Every wait of the migration kernels for a trace-row copy is bounded.  With
PSTM_CUDA_INJECT_FAULT=wait the launch leaves the first chunks' copies
unissued, so nothing completes the phase the kernel waits for; the wait gives
up after a few polls, the kernel raises its error bit and returns, and the host
reports PSTM_ERR_TIMEOUT.  No GPU fault is involved: the kernel exits normally
and the context stays usable, which the second half of each test checks
against the oracle.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _fresh_output(case):
    from pstm_b200.base import OutputTile
    out = case.output
    return OutputTile(image=np.zeros_like(out.image), fold=np.zeros_like(out.fold), x_axis=out.x_axis,
                      y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)


@pytest.fixture
def inject_wait(monkeypatch):
    def on():
        monkeypatch.setenv("PSTM_CUDA_INJECT_FAULT", "wait")

    def off():
        monkeypatch.delenv("PSTM_CUDA_INJECT_FAULT", raising=False)
    yield on, off
    off()


def _oracle(case):
    from oracle import oracle
    ref = _fresh_output(case)
    oracle.migrate(case.traces, ref, case.velocity, case.config)
    return ref


@pytest.mark.parametrize("segment_mb", [None, "1"])
def test_host_path_reports_timeout_then_recovers(cuda_kernel_factory, inject_wait, monkeypatch, segment_mb):
    """Per-tile grid launch and the segment-major persistent launch."""
    from pstm_b200 import _native as nat
    from pstm_b200 import workloads
    on, off = inject_wait
    if segment_mb:
        monkeypatch.setenv("PSTM_CUDA_SEGMENT_MB", segment_mb)   # read when the context is created
    case = workloads.config1(n_traces=4096, nx=8, ny=8, nt=500)
    k = cuda_kernel_factory(case.config)
    on()
    with pytest.raises(nat.PstmCudaError) as ei:
        k.migrate_tile(case.traces, _fresh_output(case), case.velocity)
    assert ei.value.code == nat.ERR_TIMEOUT
    assert "partial sums" in str(ei.value)
    off()
    out = _fresh_output(case)
    k.migrate_tile(case.traces, out, case.velocity)
    ref = _oracle(case)
    np.testing.assert_array_equal(out.fold, ref.fold)
    assert rel_l2(out.image, ref.image) <= 1e-5


def test_device_path_reports_timeout_at_synchronize(cuda_kernel_factory, inject_wait):
    import torch
    from pstm_b200 import _native as nat
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile
    on, off = inject_wait
    case = workloads.config1(n_traces=2048, nx=6, ny=6, nt=500)
    k = cuda_kernel_factory(case.config)
    tb = case.traces
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    from pstm_b200.base import TraceBlock
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    out = case.output

    def dev_out():
        return OutputTile(image=torch.zeros(out.image.shape, dtype=torch.float64, device="cuda"),
                          fold=torch.zeros(out.fold.shape, dtype=torch.int32, device="cuda"),
                          x_axis=dev(out.x_axis), y_axis=dev(out.y_axis), t_axis_ms=dev(out.t_axis_ms))
    from pstm_b200.base import VelocitySlice
    vel = VelocitySlice(vrms=dev(case.velocity.vrms), is_1d=True)
    on()
    k.migrate_tile(dtb, dev_out(), vel)   # asynchronous: the launch itself succeeds
    with pytest.raises(nat.PstmCudaError) as ei:
        k.synchronize()
    assert ei.value.code == nat.ERR_TIMEOUT
    off()
    o = dev_out()
    k.migrate_tile(dtb, o, vel)
    k.synchronize()
    ref = _oracle(case)
    np.testing.assert_array_equal(o.fold.cpu().numpy(), ref.fold)
    assert rel_l2(o.image.cpu().numpy(), ref.image) <= 1e-5
