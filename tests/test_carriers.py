"""The carriers of the drop-in boundary (pstm_b200.base), checked as the
reference checks its own (tests/test_kernels.py:14-70 of the reference):
trace block sizes, offsets and validation, output tile sizes and reset,
KernelConfig defaults, and the backend's name and its "not initialized"
error before ``initialize`` (numba_cpu_optimized.py:555-556)."""
from __future__ import annotations

import numpy as np
import pytest

from pstm_b200.base import KernelConfig, create_output_tile, create_trace_block


def test_trace_block_sizes_offsets_and_validation():
    rng = np.random.default_rng(0)
    b = create_trace_block(rng.standard_normal((100, 500)).astype(np.float32), np.zeros(100), np.zeros(100),
                           np.linspace(0, 1000, 100), np.zeros(100), sample_rate_ms=2.0)
    assert (b.n_traces, b.n_samples) == (100, 500)
    o = create_trace_block(np.zeros((10, 100), np.float32), np.zeros(10), np.zeros(10), np.full(10, 100.0),
                           np.zeros(10), sample_rate_ms=2.0)
    np.testing.assert_array_almost_equal(o.offset, 100.0)
    np.testing.assert_array_equal(o.midpoint_x, 50.0)
    assert o.validate() == []
    bad = create_trace_block(np.zeros((10, 100), np.float32), np.zeros(10), np.zeros(10), np.zeros(10),
                             np.zeros(10), sample_rate_ms=2.0)
    bad.source_x = np.zeros(9)
    assert bad.validate()


def test_output_tile_sizes_and_reset():
    t = create_output_tile(x_min=0, x_max=100, dx=10, y_min=0, y_max=100, dy=10, t_min_ms=0, t_max_ms=1000, dt_ms=2)
    assert (t.nx, t.ny, t.nt) == (11, 11, 501)
    t = create_output_tile(0, 100, 25, 0, 100, 25, 0, 100, 2)
    t.image[:] = 1.0
    t.fold[:] = 10
    t.reset()
    assert np.all(t.image == 0.0) and np.all(t.fold == 0)


def test_kernel_config_defaults():
    c = KernelConfig()
    assert c.max_aperture_m == 5000.0
    assert c.apply_spreading is True and c.apply_obliquity is True
    assert c.interpolation_method == "linear"


def test_backend_name_and_uninitialized_error():
    from pstm_b200.cuda_kernel import CudaKernel
    k = CudaKernel()
    assert isinstance(k.name, str) and k.name
    b = create_trace_block(np.zeros((2, 10), np.float32), np.zeros(2), np.zeros(2), np.ones(2), np.ones(2),
                           sample_rate_ms=2.0)
    t = create_output_tile(0, 10, 10, 0, 10, 10, 0, 10, 2)
    from pstm_b200.base import VelocitySlice
    with pytest.raises(RuntimeError, match="not initialized"):
        k.migrate_tile(b, t, VelocitySlice(vrms=np.full(t.nt, 2000.0), is_1d=True))
