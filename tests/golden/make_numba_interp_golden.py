"""Golden images of the reference's NumbaKernel with its trace interpolators.

Runs ``NumbaKernel.migrate_tile`` of ``pstm/kernels/numba_cpu.py`` (the
reference backend that honours ``KernelConfig.interpolation_method``,
numba_cpu.py:220-364, 584-664) from the reference checkout on one seeded
case-1 subset (250 traces cut to 300 samples, 3 x 3 pillars, 300 output
times) -- trace weights, time-varying aperture, taper, spreading and
obliquity, 2-D fold -- once per non-linear method, and stores inputs and
outputs in ``tests/golden/interp_numba_kernel.npz``.  Run once in a container
that has the reference at REF (``PSTM_REFERENCE``, default the installed reference in ``baseline/_ref``):

    NUMBA_CACHE_DIR=/tmp/numba PYTHONDONTWRITEBYTECODE=1 \\
        python tests/golden/make_numba_interp_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "interp_numba_kernel.npz")
METHODS = ["nearest", "cubic", "sinc4", "sinc8", "sinc16", "lanczos3", "lanczos5"]
CFG = dict(max_aperture_m=1000.0, min_aperture_m=500.0, max_dip_degrees=60.0, taper_fraction=0.15,
           apply_spreading=True, apply_obliquity=True, aa_enabled=False)


def main():
    sys.dont_write_bytecode = True
    sys.path.insert(0, REF)
    sys.path.insert(1, ROOT)
    from pstm.kernels import base as rb
    from pstm.kernels.numba_cpu import NumbaKernel
    from pstm_b200 import workloads
    case = workloads.config1(seed=21, n_traces=250, nx=64, ny=64, nt=300)
    tb = case.traces
    amps = np.ascontiguousarray(np.asarray(tb.amplitudes, np.float32)[:, :300])
    rng = np.random.default_rng(4)
    w = rng.uniform(0.5, 1.5, amps.shape[0])
    x, y = case.output.x_axis[30:33], case.output.y_axis[28:31]
    t = case.output.t_axis_ms
    vrms = np.asarray(case.velocity.vrms, np.float64)
    res = dict(amplitudes=amps, source_x=tb.source_x, source_y=tb.source_y,
               receiver_x=tb.receiver_x, receiver_y=tb.receiver_y, weights=w, sample_rate_ms=tb.sample_rate_ms,
               x_axis=x, y_axis=y, t_axis_ms=t, vrms=vrms, **{k: v for k, v in CFG.items()})
    for m in METHODS:
        rtb = rb.create_trace_block(amps, tb.source_x, tb.source_y,
                                    tb.receiver_x, tb.receiver_y, sample_rate_ms=tb.sample_rate_ms, weights=w)
        out = rb.OutputTile(image=np.zeros((len(x), len(y), len(t))), fold=np.zeros((len(x), len(y)), np.int32),
                            x_axis=x, y_axis=y, t_axis_ms=t)
        cfg = rb.KernelConfig(interpolation_method=m, **CFG)
        k = NumbaKernel()
        k.initialize(cfg)
        k.migrate_tile(rtb, out, rb.VelocitySlice(vrms=vrms, is_1d=True), cfg)
        res[f"{m}_image"], res[f"{m}_fold"] = out.image, out.fold
        print(f"{m}: |image| max {np.abs(out.image).max():.3e}, fold max {out.fold.max()}")
    np.savez_compressed(OUT, **res)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
