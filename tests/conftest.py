"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_files(prefix="numba_"):
    return sorted(glob.glob(os.path.join(GOLDEN, f"{prefix}*.npz")))


def load_golden_case(path):
    """(traces, output, velocity, config, expected_image, expected_fold) from a fixture."""
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    z = np.load(path)
    w = z["weights"] if bool(z["has_weights"]) else None
    tb = create_trace_block(z["amplitudes"], z["source_x"], z["source_y"], z["receiver_x"], z["receiver_y"],
                            sample_rate_ms=float(z["sample_rate_ms"]), start_time_ms=float(z["start_time_ms"]),
                            weights=w)
    x, y, t = z["x_axis"], z["y_axis"], z["t_axis_ms"]
    fold = np.zeros(z["fold"].shape, np.int32)
    out = OutputTile(image=np.zeros((len(x), len(y), len(t))), fold=fold, x_axis=x, y_axis=y, t_axis_ms=t)
    vt = z["vel_t_axis"] if bool(z["has_vel_t_axis"]) else None
    vel = VelocitySlice(vrms=z["vrms"], is_1d=True, t_axis_ms=vt)
    cfg = KernelConfig(max_aperture_m=float(z["max_aperture_m"]), min_aperture_m=float(z["min_aperture_m"]),
                       max_dip_degrees=float(z["max_dip_degrees"]), taper_fraction=float(z["taper_fraction"]),
                       apply_spreading=bool(z["apply_spreading"]), apply_obliquity=bool(z["apply_obliquity"]),
                       aa_enabled=False)
    return tb, out, vel, cfg, z["image"], z["fold"]


def interp_velocity(vel, t_axis):
    """The reference's np.interp of a 1-D velocity onto the output axis."""
    from pstm_b200.base import VelocitySlice
    v = np.asarray(vel.vrms, np.float64)
    if len(v) != len(t_axis):
        vt = t_axis if vel.t_axis_ms is None else vel.t_axis_ms
        v = np.interp(t_axis, vt, v)
    return VelocitySlice(vrms=v, is_1d=True)


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda_kernel_factory():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from pstm_b200 import build
    build.build()
    from pstm_b200.cuda_kernel import CudaKernel
    made = []

    def make(config, **kw):
        k = CudaKernel(**kw)
        k.initialize(config)
        made.append(k)
        return k
    yield make
    for k in made:
        k.cleanup()
