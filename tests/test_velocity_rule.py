"""The Metal host's lateral-velocity rule (metal_compiled.py:631-664) behind
``CudaKernel(velocity_mode="auto")``: the 3-D cube only when max |v - v_centre|
/ mean(v_centre) exceeds 5 %, else the centre pillar for every pillar.  Host
logic, checked on CPU for NumPy arrays and torch tensors."""
from __future__ import annotations

import numpy as np
import pytest

from pstm_b200.cuda_kernel import lateral_velocity_choice


def _cube(dev):
    v = np.full((5, 4, 30), 2000.0)
    v[..., :] += np.linspace(0.0, 1000.0, 30)           # same trend in every pillar
    v[0, 0, 7] += dev * v[2, 2, :].mean()                # one corner sample off by `dev`
    return v


@pytest.mark.parametrize("lib", ["numpy", "torch"])
@pytest.mark.parametrize("dev,is3d", [(0.0, False), (0.049, False), (0.05, False), (0.0501, True), (0.3, True)])
def test_threshold(dev, is3d, lib):
    v = _cube(dev)
    if lib == "torch":
        import torch
        v = torch.as_tensor(v)
    out, use3d = lateral_velocity_choice(v)
    assert use3d == is3d
    got = np.asarray(out)
    if is3d:
        assert got.shape == (5, 4, 30) and np.array_equal(got, np.asarray(v))
    else:
        assert got.shape == (30,) and np.array_equal(got, np.asarray(v)[2, 2, :])
