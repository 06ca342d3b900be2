"""The precision form's trace format on the host (CPU): FP16 with one
power-of-two scale per trace, carried by the trace weight."""
from __future__ import annotations

import numpy as np


def test_scaled_f16_range_exactness_and_rounding():
    from pstm_b200.cuda_kernel import scaled_f16
    rng = np.random.default_rng(0)
    levels = np.logspace(-20, 20, 64).astype(np.float32)
    a = rng.standard_normal((64, 500)).astype(np.float32) * levels[:, None]
    a[3] = 0.0
    h, inv = scaled_f16(a)
    assert h.dtype == np.float16 and np.isfinite(h).all()
    peak = np.abs(h.astype(np.float32)).max(axis=1)
    live = np.arange(64) != 3
    # every nonzero trace's largest |amplitude| lands in [2^13, 2^14] (rounding may reach 2^14)
    assert (peak[live] >= 2.0 ** 13).all() and (peak[live] <= 2.0 ** 14).all()
    assert inv[3] == 1.0 and not h[3].any()
    # the scales are powers of two, so amplitude x weight is the FP32 trace up to FP16 rounding
    assert np.all(np.frexp(inv)[0] == 0.5)
    back = h.astype(np.float64) * inv[:, None]
    big = (np.abs(a) >= np.abs(a).max(axis=1, keepdims=True) * 2.0 ** -10) & live[:, None]
    rel = np.abs(back - a)[big] / np.abs(a)[big]
    assert rel.max() <= 2.0 ** -11


def test_to_f16_panel_host_weights():
    from pstm_b200 import workloads
    from pstm_b200.cuda_kernel import CudaKernel, scaled_f16
    case = workloads.config1(n_traces=200, nx=4, ny=4, nt=50)
    tb = case.traces
    k = CudaKernel(trace_dtype="f16")   # no device needed for host arrays
    p = k.to_f16_panel(tb)
    h, inv = scaled_f16(tb.amplitudes)
    np.testing.assert_array_equal(p.amplitudes.view(np.uint16), h.view(np.uint16))
    np.testing.assert_array_equal(p.weights, inv)
    assert p.source_x is tb.source_x
