"""Randomised configurations, oracle against the reference's own CPU kernel
(``OptimizedNumbaKernel``, numba_cpu_optimized.py:93-233, 545-626), run live
where the reference tree and Numba are importable (skipped elsewhere; the six
committed ``tests/golden/numba_*.npz`` cases pin the same path everywhere).
Each draw picks aperture (max and min), dip, taper (0 included), spreading and
obliquity, trace weights or none, sample rate, start time and a 2-D or 3-D
fold; band-limited traces.  The FP64 oracle must reproduce the image to 1e-12
(the reference compiles with fastmath) and the fold exactly."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle

_REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")
HERE = os.path.dirname(os.path.abspath(__file__))
# Numba caches compiled functions; keep that cache inside the repository's own pytest cache
os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(os.path.dirname(HERE), ".pytest_cache", "numba"))


@pytest.fixture(scope="module")
def numba_kernel():
    if not os.path.isdir(os.path.join(REF, "pstm", "kernels")):
        pytest.skip("the reference tree is not present")
    pytest.importorskip("numba")
    sys.dont_write_bytecode = True
    if REF not in sys.path:
        sys.path.append(REF)
    from pstm.kernels import base as rb
    from pstm.kernels.numba_cpu_optimized import OptimizedNumbaKernel
    return rb, OptimizedNumbaKernel


@pytest.mark.parametrize("seed", range(10))
def test_random_configuration(seed, numba_kernel):
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    rb, Kernel = numba_kernel
    oracle.build()
    rng = np.random.default_rng(seed)
    n, ns, nt = 150, 300, 120
    s, r = rng.uniform(0, 1500, (n, 2)), rng.uniform(0, 1500, (n, 2))
    tw = np.arange(-25, 26) * 0.004
    ricker = (1 - 2 * (np.pi * 25 * tw) ** 2) * np.exp(-(np.pi * 25 * tw) ** 2)
    amps = np.array([np.convolve(x, ricker, mode="same") for x in rng.standard_normal((n, ns))], np.float32)
    w = rng.uniform(0.5, 1.5, n) if rng.random() < 0.5 else None
    dt, t_start = float(rng.choice([2.0, 4.0])), float(rng.choice([0.0, 8.0, 40.0]))
    x, y = rng.uniform(300, 700) + 25 * np.arange(4), rng.uniform(300, 700) + 25 * np.arange(3)
    t_ms = 8.0 * np.arange(nt)
    v = 1600 + 1500 * t_ms / t_ms[-1]
    cfg = dict(max_aperture_m=float(rng.uniform(300, 1500)), min_aperture_m=float(rng.uniform(50, 300)),
               max_dip_degrees=float(rng.uniform(20, 80)),
               taper_fraction=float(rng.choice([0.0, rng.uniform(0.05, 0.4)])),
               apply_spreading=bool(rng.random() < 0.7), apply_obliquity=bool(rng.random() < 0.7), aa_enabled=False)
    fold_shape = (4, 3) if rng.random() < 0.5 else (4, 3, nt)
    ref = rb.OutputTile(image=np.zeros((4, 3, nt)), fold=np.zeros(fold_shape, np.int32), x_axis=x, y_axis=y,
                        t_axis_ms=t_ms)
    k = Kernel()
    k.initialize(rb.KernelConfig(**cfg))
    k.migrate_tile(rb.create_trace_block(amps, s[:, 0], s[:, 1], r[:, 0], r[:, 1], sample_rate_ms=dt,
                                         start_time_ms=t_start, weights=w), ref, rb.VelocitySlice(vrms=v, is_1d=True))
    out = OutputTile(image=np.zeros((4, 3, nt)), fold=np.zeros(fold_shape, np.int32), x_axis=x, y_axis=y,
                     t_axis_ms=t_ms)
    oracle.migrate(create_trace_block(amps, s[:, 0], s[:, 1], r[:, 0], r[:, 1], sample_rate_ms=dt,
                                      start_time_ms=t_start, weights=w), out, VelocitySlice(vrms=v, is_1d=True),
                   KernelConfig(**cfg))
    np.testing.assert_array_equal(out.fold, ref.fold)
    assert np.abs(ref.image).max() > 0
    assert rel_l2(out.image, ref.image) <= 1e-12
