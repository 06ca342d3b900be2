"""Fixtures of the reference's Metal compute shaders, run on the CPU.

Builds ``oracle/_ref/libpstm_metal_ref.so`` -- the shaders
``pstm/metal/shaders/pstm_migration.metal``, ``pstm_curved_ray.metal`` and
``pstm_anisotropic_vti.metal`` of the reference at REF (``PSTM_REFERENCE``,
default the installed reference in ``baseline/_ref``), compiled unchanged as C++ by ``oracle/Makefile``'s ``ref``
target -- runs its kernels and helpers on seeded inputs and writes their
inputs and outputs to ``tests/golden/metal_kernels.npz``; every kernel runs in
its scalar form and in its ``_simd`` form (the Metal backend's default).  Run it in a
container that has the reference:

    PSTM_REFERENCE=/path/to/reference python tests/golden/make_metal_golden.py

A sixth run is the time-variant shader (pstm_migrate_time_variant) at the
windows of a seeded frequency table, 3-D velocity, AA on.  The tests read
only the .npz.  All inputs are FP32-exact (the shaders take FP32), so the
FP64 oracle sees the same numbers.  The aperture is one constant
(min_aperture = max_aperture): the Metal host's per-time aperture law is not
under test here (the straight-ray law is pinned to the reference's Numba
kernel by make_golden.py).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.environ.get("PSTM_REFERENCE") or os.path.join(_REPO, "baseline", "_ref")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "metal_kernels.npz")

# one entry per kernel run: kind, velocity ("1d" | "3d"), grid ("axes" | "rotated"),
# t_start_ms, AA, spreading, obliquity, curved (v0, k), eta ("1d" | constant)
CASES = [
    ("straight_3dvel_aa", "straight", "3d", "axes", 0.0, 1, 1, 1, (0.0, 0.0), None),
    ("straight_rotated_tstart", "straight", "1d", "rotated", 40.0, 0, 1, 0, (0.0, 0.0), None),
    ("curved_aa", "curved", "1d", "axes", 0.0, 1, 1, 1, (1800.0, 0.6), None),
    ("vti_eta1d_aa", "vti", "1d", "axes", 0.0, 1, 1, 1, (0.0, 0.0), "1d"),
    ("vti_eta_const", "vti", "1d", "rotated", 0.0, 0, 1, 1, (0.0, 0.0), 0.1),
]
APERTURE, TAPER, DX, DT_MS, NX, NY, NT, NS = 900.0, 0.1, 25.0, 4.0, 6, 5, 120, 300


def inputs():
    from pstm_b200 import workloads
    case = workloads.config1(n_traces=200, nx=NX, ny=NY, nt=NT)
    tb, out = case.traces, case.output
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    rng = np.random.default_rng(3)
    t_ms = np.asarray(out.t_axis_ms[:NT], np.float64)
    v1 = f32(np.asarray(case.velocity.vrms, np.float64)[:NT])
    X, Y = np.meshgrid(np.asarray(out.x_axis, np.float64), np.asarray(out.y_axis, np.float64), indexing="ij")
    ang = 0.35
    return dict(
        amps=f32(np.asarray(tb.amplitudes)[:, :NS]), sx=f32(tb.source_x), sy=f32(tb.source_y),
        rx=f32(tb.receiver_x), ry=f32(tb.receiver_y), t_ms=t_ms, v1=v1,
        v3=f32(v1[None, None, :] * (1 + 0.05 * rng.standard_normal((NX, NY, 1)))),
        eta1=f32(0.3 * t_ms / 1000.0), X=f32(X), Y=f32(Y),
        Xr=f32(700 + (X - 700) * np.cos(ang) - (Y - 700) * np.sin(ang)),
        Yr=f32(700 + (X - 700) * np.sin(ang) + (Y - 700) * np.cos(ang)))


def run_case(mr, d, spec, simd=False):
    name, kind, vel, grid, t0ms, aa, spr, obl, (v0, k), eta = spec
    X, Y = (d["X"], d["Y"]) if grid == "axes" else (d["Xr"], d["Yr"])
    return mr.migrate(kind, d["amps"], d["sx"], d["sy"], d["rx"], d["ry"], X, Y, d["t_ms"],
                      d["v3"] if vel == "3d" else d["v1"], aperture_m=APERTURE, taper=TAPER, dx=DX, dy=DX,
                      dt_ms=DT_MS, t_start_ms=t0ms, spreading=bool(spr), obliquity=bool(obl), aa=bool(aa),
                      v0=v0, k=k, eta=d["eta1"] if eta == "1d" else None,
                      eta_constant=eta if isinstance(eta, float) else 0.0, simd=simd)


TV_TABLE = ([0.0, 150.0, 300.0, 476.0], [80.0, 60.0, 25.0, 12.0])   # (ms, Hz)


def tv_windows():
    """Time-variant windows over the case's output axis at the 4 ms base rate."""
    from pstm_b200 import time_variant as tvm
    table = tvm.FrequencyTimeTable(times_ms=TV_TABLE[0], frequencies_hz=TV_TABLE[1])
    return tvm.compute_time_windows(0.0, (NT - 1) * DT_MS + DT_MS, DT_MS, table)


def run_tv(mr, d):
    return mr.migrate_time_variant(d["amps"], d["sx"], d["sy"], d["rx"], d["ry"], d["X"], d["Y"], d["v3"],
                                   tv_windows(), aperture_m=APERTURE, taper=TAPER, dx=DX, dy=DX, dt_ms=DT_MS)


def helper_rows(mr):
    """Curved-ray and VTI two-leg traveltimes at seeded (t0, h_s, h_r, v, eta)."""
    rng = np.random.default_rng(11)
    n = 400
    t0 = rng.uniform(0.0, 3.0, n).astype(np.float32)
    hs, hr = (rng.uniform(0.0, 3000.0, n).astype(np.float32) for _ in range(2))
    v = rng.uniform(1500.0, 4000.0, n).astype(np.float32)
    eta = rng.uniform(0.0, 0.2, n).astype(np.float32)
    v0, k = np.float32(1700.0), np.float32(0.55)
    z = mr.time_to_depth(t0 / np.float32(2.0), np.full(n, v0), np.full(n, k))
    return dict(h_t0=t0, h_hs=hs, h_hr=hr, h_v=v, h_eta=eta, h_v0=v0, h_k=k, h_z=z,
                h_curved=mr.curved_dsr(hs, hr, z, np.full(n, v0), np.full(n, k)),
                h_vti=mr.vti_dsr(t0, hs, hr, v, eta))


def main():
    from oracle import metal_ref as mr
    if mr.build(REF) is None:
        sys.exit(f"no reference tree at {REF}")
    d = inputs()
    res = dict(d)
    for spec in CASES:
        img, fold = run_case(mr, d, spec)
        res[f"{spec[0]}_image"], res[f"{spec[0]}_fold"] = img, fold
        res[f"{spec[0]}_simd_image"], res[f"{spec[0]}_simd_fold"] = run_case(mr, d, spec, simd=True)
    res["tv_image"], res["tv_fold"] = run_tv(mr, d)
    res.update(helper_rows(mr))
    np.savez_compressed(OUT, **res)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
