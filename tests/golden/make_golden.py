"""Generate golden fixtures by running the reference implementation.

Run in a container where the reference project is importable (it is read
from REF: ``PSTM_REFERENCE``, default the installed reference in ``baseline/_ref``); the tests read only its output.  Writes
``*.npz`` next to this file:

* ``numba_*.npz``   inputs and outputs of the reference's registered CPU
  backend ``OptimizedNumbaKernel.migrate_tile``
  (pstm/kernels/numba_cpu_optimized.py:545-626) on small seeded cases,
  including the edge cases its own tests exercise (single trace, traces far
  outside the aperture; tests/test_kernels.py:111-150);
* ``traveltime_curved_vti.npz``  the reference's Python curved-ray and VTI
  traveltimes (pstm/algorithm/curved_ray.py:287-316,
  pstm/algorithm/anisotropy_vti.py:148-220) on seeded random inputs.

    NUMBA_CACHE_DIR=/tmp/nb PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")
sys.path.insert(0, REF)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pstm.kernels import base as rb  # noqa: E402
from pstm.kernels.numba_cpu_optimized import OptimizedNumbaKernel  # noqa: E402
from pstm.algorithm import curved_ray as rcr  # noqa: E402
from pstm.algorithm import anisotropy_vti as rvti  # noqa: E402

from pstm_b200 import workloads  # noqa: E402


def run_numba(name, amps, sx, sy, rx, ry, dt_ms, t0_ms, x, y, t_axis, vrms, cfg_kw,
              weights=None, fold_2d=False, vel_t_axis=None):
    tb = rb.create_trace_block(amps, sx, sy, rx, ry, sample_rate_ms=dt_ms, start_time_ms=t0_ms,
                               weights=weights)
    nx, ny, nt = len(x), len(y), len(t_axis)
    fold = np.zeros((nx, ny) if fold_2d else (nx, ny, nt), np.int32)
    out = rb.OutputTile(image=np.zeros((nx, ny, nt)), fold=fold, x_axis=x, y_axis=y, t_axis_ms=t_axis)
    vel = rb.VelocitySlice(vrms=vrms, is_1d=True, t_axis_ms=vel_t_axis)
    cfg = rb.KernelConfig(**cfg_kw)
    k = OptimizedNumbaKernel()
    k.initialize(cfg)
    k.migrate_tile(tb, out, vel)
    np.savez_compressed(
        os.path.join(HERE, f"numba_{name}.npz"),
        amplitudes=np.asarray(amps, np.float32), source_x=sx, source_y=sy, receiver_x=rx, receiver_y=ry,
        weights=np.array([]) if weights is None else weights, has_weights=weights is not None,
        sample_rate_ms=dt_ms, start_time_ms=t0_ms, x_axis=x, y_axis=y, t_axis_ms=t_axis, vrms=vrms,
        vel_t_axis=np.array([]) if vel_t_axis is None else vel_t_axis, has_vel_t_axis=vel_t_axis is not None,
        max_aperture_m=cfg.max_aperture_m, min_aperture_m=cfg.min_aperture_m,
        max_dip_degrees=cfg.max_dip_degrees, taper_fraction=cfg.taper_fraction,
        apply_spreading=cfg.apply_spreading, apply_obliquity=cfg.apply_obliquity,
        image=out.image, fold=out.fold,
    )
    print(f"numba_{name}: image |max| {np.abs(out.image).max():.3e} fold max {out.fold.max()}")


def main():
    # 1. config-1 geometry, 512 traces, 8x8 pillars around the first diffractor
    case = workloads.config1(seed=11, n_traces=512)
    tb = case.traces
    c1 = dict(max_aperture_m=1000.0, min_aperture_m=500.0, max_dip_degrees=60.0, taper_fraction=0.1,
              apply_spreading=True, apply_obliquity=True, aa_enabled=False)
    x, y = case.output.x_axis[28:36], case.output.y_axis[28:36]
    run_numba("c1_subset", tb.amplitudes, tb.source_x, tb.source_y, tb.receiver_x, tb.receiver_y,
              4.0, 0.0, x, y, case.output.t_axis_ms, case.velocity.vrms, c1)

    rng = np.random.default_rng(5)
    # 2. trace weights, wide taper, other dip/min aperture, non-square tile, 2 ms
    n, ns = 300, 400
    sx, sy = rng.uniform(0, 800, n), rng.uniform(0, 800, n)
    rx, ry = rng.uniform(0, 800, n), rng.uniform(0, 800, n)
    amps = rng.standard_normal((n, ns)).astype(np.float32)
    w = rng.uniform(0.2, 2.0, n)
    x, y = 300 + 20.0 * np.arange(5), 250 + 15.0 * np.arange(7)
    t_axis = 2.0 * np.arange(350)
    vrms = np.linspace(1600.0, 3200.0, 350)
    run_numba("weights_taper", amps, sx, sy, rx, ry, 2.0, 0.0, x, y, t_axis, vrms,
              dict(max_aperture_m=600.0, min_aperture_m=200.0, max_dip_degrees=35.0, taper_fraction=0.3,
                   apply_spreading=True, apply_obliquity=True, aa_enabled=False), weights=w)

    # 3. start time > 0, spreading off, velocity on a coarser axis (np.interp path), 2-D fold
    t_axis = 100.0 + 4.0 * np.arange(120)
    vt = np.array([0.0, 300.0, 700.0])
    vv = np.array([1800.0, 2100.0, 2600.0])
    run_numba("start_time_interp", amps[:, :200], sx, sy, rx, ry, 4.0, 60.0, x, y, t_axis, vv,
              dict(max_aperture_m=700.0, min_aperture_m=300.0, max_dip_degrees=45.0, taper_fraction=0.1,
                   apply_spreading=False, apply_obliquity=True, aa_enabled=False),
              fold_2d=True, vel_t_axis=vt)

    # 4. hard aperture edge (taper 0), obliquity off
    run_numba("taper0", amps, sx, sy, rx, ry, 2.0, 0.0, x, y, 2.0 * np.arange(200),
              np.full(200, 2200.0),
              dict(max_aperture_m=350.0, min_aperture_m=350.0, max_dip_degrees=45.0, taper_fraction=0.0,
                   apply_spreading=True, apply_obliquity=False, aa_enabled=False))

    # 5. single trace (tests/test_kernels.py:111-127)
    run_numba("single_trace", rng.standard_normal((1, 100)).astype(np.float32), np.array([0.0]),
              np.array([0.0]), np.array([100.0]), np.array([0.0]), 2.0, 0.0,
              np.arange(0, 101, 25.0), np.arange(-50, 51, 25.0), 2.0 * np.arange(51), np.full(51, 2000.0),
              dict(max_aperture_m=500.0))

    # 6. traces far outside the aperture (tests/test_kernels.py:129-150): fold 0, image 0
    run_numba("far_traces", rng.standard_normal((10, 100)).astype(np.float32), np.full(10, 10000.0),
              np.full(10, 10000.0), np.full(10, 10100.0), np.full(10, 10000.0), 2.0, 0.0,
              np.arange(0, 101, 25.0), np.arange(0, 101, 25.0), 2.0 * np.arange(51), np.full(51, 2000.0),
              dict(max_aperture_m=100.0))

    # 7. traveltimes of the reference's Python curved-ray / VTI formulas
    m = 400
    t0 = rng.uniform(0.0, 3.0, m)
    t0[:5] = 0.0
    hs, hr = rng.uniform(0, 4000, m), rng.uniform(0, 4000, m)
    v = rng.uniform(1500, 4000, m)
    eta = rng.uniform(0.0, 0.2, m)
    v0 = rng.uniform(1400, 2200, m)
    k = rng.uniform(0.0, 1.5, m)
    k[5:10] = 0.0
    Tc = np.array([rcr.curved_ray_dsr_traveltime(t0[i], hs[i], hr[i], v0[i], k[i]) for i in range(m)])
    Tv = np.array([rvti.vti_dsr_traveltime(t0[i], hs[i], hr[i], v[i], eta[i]) for i in range(m)])
    np.savez_compressed(os.path.join(HERE, "traveltime_curved_vti.npz"), t0=t0, hs=hs, hr=hr, v=v,
                        eta=eta, v0=v0, k=k, T_curved=Tc, T_vti=Tv)
    print("traveltime_curved_vti: ok")


if __name__ == "__main__":
    main()
