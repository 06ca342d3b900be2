"""Whole migrations with the non-linear trace interpolators against the
reference's own NumbaKernel (numba_cpu.py:220-364), whose images for nearest,
cubic, windowed sinc 4/8/16 and Lanczos 3/5 are committed in
``tests/golden/interp_numba_kernel.npz`` by ``make_numba_interp_golden.py``
(trace weights, time-varying aperture, taper, spreading, obliquity, 2-D fold).
The FP64 oracle must reproduce them to 1e-10 (the reference compiles with
fastmath), the CUDA interpolation kernel to 1e-9, the folds exactly."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "interp_numba_kernel.npz")
METHODS = ["nearest", "cubic", "sinc4", "sinc8", "sinc16", "lanczos3", "lanczos5"]


def _case(method):
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    d = dict(np.load(FIXTURE))
    tb = create_trace_block(d["amplitudes"], d["source_x"], d["source_y"], d["receiver_x"], d["receiver_y"],
                            sample_rate_ms=float(d["sample_rate_ms"]), weights=d["weights"])
    out = OutputTile(image=np.zeros(d[f"{method}_image"].shape), fold=np.zeros(d[f"{method}_fold"].shape, np.int32),
                     x_axis=d["x_axis"], y_axis=d["y_axis"], t_axis_ms=d["t_axis_ms"])
    cfg = KernelConfig(max_aperture_m=float(d["max_aperture_m"]), min_aperture_m=float(d["min_aperture_m"]),
                       max_dip_degrees=float(d["max_dip_degrees"]), taper_fraction=float(d["taper_fraction"]),
                       apply_spreading=bool(d["apply_spreading"]), apply_obliquity=bool(d["apply_obliquity"]),
                       aa_enabled=False, interpolation_method=method)
    return tb, out, VelocitySlice(vrms=d["vrms"], is_1d=True), cfg, d[f"{method}_image"], d[f"{method}_fold"]


@pytest.mark.parametrize("method", METHODS)
def test_oracle_matches_numba_kernel(method):
    oracle.build()
    tb, out, vel, cfg, img, fold = _case(method)
    oracle.migrate(tb, out, vel, cfg)
    np.testing.assert_array_equal(out.fold, fold)
    assert np.abs(img).max() > 0
    assert rel_l2(out.image, img) <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("method", METHODS)
def test_cuda_matches_numba_kernel(method, cuda_kernel_factory):
    tb, out, vel, cfg, img, fold = _case(method)
    k = cuda_kernel_factory(cfg)
    k.migrate_tile(tb, out, vel, cfg)
    np.testing.assert_array_equal(out.fold, fold)
    assert rel_l2(out.image, img) <= 1e-9
