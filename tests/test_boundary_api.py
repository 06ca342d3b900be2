"""The drop-in boundary against the reference's own API (CPU).

Where the reference tree is importable (``PSTM_REFERENCE``, default
the installed reference in ``baseline/_ref``; skipped elsewhere), its carriers (``pstm/kernels/base.py``:
TraceBlock, OutputTile, VelocitySlice, KernelConfig, KernelMetrics) must have
every field here under the same name with the same default, its
``KernelCapability`` members must exist here, ``CudaKernel`` must provide every
method of its ``MigrationKernel`` protocol (base.py:290-318) and the optional
methods the executor looks up with ``hasattr`` (executor.py:1691-1745), and
``create_trace_block`` must form the same offsets and midpoints."""
from __future__ import annotations

import dataclasses
import os
import sys

import numpy as np
import pytest

_REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")


@pytest.fixture(scope="module")
def rb():
    if not os.path.isdir(os.path.join(REF, "pstm", "kernels")):
        pytest.skip("the reference tree is not present")
    sys.dont_write_bytecode = True   # the reference tree is read-only
    if REF not in sys.path:
        sys.path.append(REF)
    from pstm.kernels import base
    return base


@pytest.mark.parametrize("name", ["TraceBlock", "OutputTile", "VelocitySlice", "KernelConfig", "KernelMetrics"])
def test_carrier_fields_and_defaults(name, rb):
    from pstm_b200 import base as ours
    theirs = {f.name: f for f in dataclasses.fields(getattr(rb, name))}
    mine = {f.name: f for f in dataclasses.fields(getattr(ours, name))}
    missing = sorted(set(theirs) - set(mine))
    assert not missing, f"{name} lacks {missing}"
    for n, f in theirs.items():
        if f.default is not dataclasses.MISSING:
            assert mine[n].default == f.default, f"{name}.{n}: default {mine[n].default!r} != {f.default!r}"


def test_capabilities_and_protocol(rb):
    from pstm_b200 import base as ours
    from pstm_b200.cuda_kernel import CudaKernel
    assert set(rb.KernelCapability.__members__) <= set(ours.KernelCapability.__members__)
    for m in ("name", "capabilities", "initialize", "migrate_tile", "synchronize", "cleanup",
              "migrate_tile_curved_ray", "migrate_tile_vti", "migrate_tile_time_variant"):
        assert hasattr(CudaKernel, m), m
    # with the reference importable, the kernel reports the reference's own enum
    # members, so `KernelCapability.X in kernel.capabilities` holds in its code
    caps = CudaKernel().capabilities
    assert caps and caps <= set(rb.KernelCapability)


def test_create_trace_block_matches(rb):
    from pstm_b200.base import create_trace_block
    rng = np.random.default_rng(1)
    a = rng.standard_normal((50, 40)).astype(np.float32)
    s, r = rng.uniform(-500, 3000, (2, 50)), rng.uniform(-500, 3000, (2, 50))
    w = rng.uniform(0.5, 2.0, 50)
    mine = create_trace_block(a, s[0], s[1], r[0], r[1], sample_rate_ms=2.0, start_time_ms=8.0, weights=w)
    theirs = rb.create_trace_block(a, s[0], s[1], r[0], r[1], sample_rate_ms=2.0, start_time_ms=8.0, weights=w)
    for f in ("offset", "midpoint_x", "midpoint_y", "weights", "source_x", "receiver_y"):
        np.testing.assert_array_equal(getattr(mine, f), getattr(theirs, f))
    assert (mine.sample_rate_ms, mine.start_time_ms) == (theirs.sample_rate_ms, theirs.start_time_ms)
