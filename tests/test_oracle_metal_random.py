"""Randomised configurations, oracle against the reference's Metal shader
kernels compiled as C++ (CPU; runs where ``oracle/_ref`` is built, i.e. where
the reference tree is, and is skipped elsewhere).  Each draw picks aperture,
taper (0 included: the hard cut), AA, spreading and obliquity on or off, start
time, grid spacing, a rotated or axis grid, the curved gradient (k = 0
included: the straight-ray fallback) and eta.  Traces are band-limited noise
(white noise convolved with a 25 Hz Ricker wavelet, like seismic data), so the
shaders' FP32 sample positions cost FP32-sized errors.  The FP64 oracle must
reproduce the FP32 shader's image (relative L2 <= 5e-5; 1e-4 for curved rays,
whose FP32 log of a ratio near 1 loses more at short times) and, where the two
fold rules coincide, the curved/VTI fold: the shaders count the traces that
contribute at t0 = 0, which are the traces within the aperture when T(t0 = 0)
= 0 lands on the trace, i.e. with no start time, for VTI and for curved rays
with k != 0 (k = 0 falls back to straight rays with T = (h_s + h_r) / v0)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from oracle import metal_ref, oracle

N_DRAWS = 12
TOL = {"straight": 5e-5, "curved": 1e-4, "vti": 5e-5}


def _draw(seed):
    rng = np.random.default_rng(seed)
    n, ns, nt = 80, 250, 70
    f32 = lambda a: np.asarray(a, np.float32)
    s, r = f32(rng.uniform(0, 1500, (n, 2))), f32(rng.uniform(0, 1500, (n, 2)))
    tw = np.arange(-25, 26) * 0.004
    ricker = (1 - 2 * (np.pi * 25.0 * tw) ** 2) * np.exp(-(np.pi * 25.0 * tw) ** 2)
    amps = f32([np.convolve(row, ricker, mode="same") for row in rng.standard_normal((n, ns))])
    dx = float(rng.choice([12.5, 25.0]))
    x0, y0 = float(rng.uniform(300, 700)), float(rng.uniform(300, 700))
    X, Y = np.meshgrid(x0 + dx * np.arange(3), y0 + dx * np.arange(4), indexing="ij")
    if rng.random() < 0.5:
        a = rng.uniform(0, np.pi)
        X, Y = 700 + (X - 700) * np.cos(a) - (Y - 700) * np.sin(a), 700 + (X - 700) * np.sin(a) + (Y - 700) * np.cos(a)
    t_ms = 8.0 * np.arange(nt)
    v1 = f32(1600 + 1500 * t_ms / t_ms[-1])
    p = dict(aperture=float(rng.uniform(200, 1500)), taper=float(rng.choice([0.0, rng.uniform(0.05, 0.5)])),
             aa=bool(rng.random() < 0.6), spreading=bool(rng.random() < 0.7), obliquity=bool(rng.random() < 0.7),
             t_start=float(rng.choice([0.0, 8.0, 40.0])), v0=float(rng.uniform(1400, 2200)),
             k=float(rng.choice([0.0, rng.uniform(0.2, 1.0)])), eta=float(rng.uniform(0.0, 0.2)),
             eta1d=bool(rng.random() < 0.5))
    return amps, s, r, f32(X), f32(Y), t_ms, v1, dx, p


def _oracle(kind, amps, s, r, X, Y, t_ms, v1, dx, p):
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    f64 = lambda a: np.asarray(a, np.float64)
    tb = create_trace_block(amps, f64(s[:, 0]), f64(s[:, 1]), f64(r[:, 0]), f64(r[:, 1]), sample_rate_ms=4.0,
                            start_time_ms=p["t_start"])
    nx, ny = X.shape
    out = OutputTile(image=np.zeros((nx, ny, len(t_ms))), fold=np.zeros((nx, ny), np.int32),
                     x_axis=np.arange(nx, dtype=np.float64), y_axis=np.arange(ny, dtype=np.float64),
                     t_axis_ms=t_ms, x_grid=f64(X), y_grid=f64(Y))
    eta1 = f64(p["eta"] * t_ms / t_ms[-1])
    kt = {"straight": "straight_ray", "curved": "curved_ray", "vti": "anisotropic_vti"}[kind]
    cfg = KernelConfig(max_aperture_m=p["aperture"], min_aperture_m=p["aperture"], max_dip_degrees=45.0,
                       taper_fraction=p["taper"], aa_enabled=p["aa"], apply_spreading=p["spreading"],
                       apply_obliquity=p["obliquity"], grid_dx=dx, grid_dy=dx, aa_dominant_freq=30.0, kernel_type=kt,
                       curved_ray_enabled=kind == "curved", curved_ray_v0=p["v0"], curved_ray_k=p["k"],
                       vti_enabled=kind == "vti", vti_eta_array=eta1 if p["eta1d"] else None,
                       vti_eta_constant=0.0 if p["eta1d"] else p["eta"])
    oracle.migrate(tb, out, VelocitySlice(vrms=f64(v1), is_1d=True), cfg, kind=kt)
    return out, eta1


@pytest.mark.parametrize("kind", ["straight", "curved", "vti"])
@pytest.mark.parametrize("seed", range(N_DRAWS))
def test_random_configuration(seed, kind):
    if not metal_ref.available():
        pytest.skip("the shader library is built only where the reference tree is")
    oracle.build()
    amps, s, r, X, Y, t_ms, v1, dx, p = _draw(1000 * seed + {"straight": 1, "curved": 2, "vti": 3}[kind])
    out, eta1 = _oracle(kind, amps, s, r, X, Y, t_ms, v1, dx, p)
    img, fold = metal_ref.migrate(kind, amps, s[:, 0], s[:, 1], r[:, 0], r[:, 1], X, Y, t_ms, v1,
                                  aperture_m=p["aperture"], taper=p["taper"], dx=dx, dy=dx, dt_ms=4.0,
                                  t_start_ms=p["t_start"], spreading=p["spreading"], obliquity=p["obliquity"],
                                  aa=p["aa"], v0=p["v0"], k=p["k"], eta=eta1 if p["eta1d"] else None,
                                  eta_constant=0.0 if p["eta1d"] else p["eta"], simd=seed % 2 == 1)
    ref = img.astype(np.float64)
    if np.abs(ref).max() == 0:
        assert np.abs(out.image).max() == 0
    else:
        assert rel_l2(out.image, ref) <= TOL[kind], p
    if kind == "vti" or (kind == "curved" and p["k"] != 0.0):
        if p["t_start"] == 0.0:
            np.testing.assert_array_equal(out.fold, fold)
