"""The oracle against the reference's Metal compute shaders (CPU).

``tests/golden/metal_kernels.npz`` holds inputs and outputs of the
reference's own shader kernels -- pstm_migrate_3d (straight rays, AA, 1-D and
3-D velocity, rotated grid, start time > 0), pstm_migrate_curved_ray and
pstm_migrate_vti (eta(t) and constant eta), pstm_migrate_time_variant (at the
windows of a frequency table) -- and of their curved-ray and VTI traveltime
helpers, compiled unchanged as C++ and run on the CPU by
``tests/golden/make_metal_golden.py``.  The FP64 oracle must reproduce the
FP32 shaders' images to FP32 accuracy (relative L2 bounds below) and, for
the curved and VTI kernels, their (nx, ny) fold exactly.  The straight
kernel's fold counts contributing traces per sample (the Metal semantics);
the oracle follows the Numba fold, so only its image is compared.  Where the
shader library is built (a container with the reference), the fixture is
also regenerated and must match bit for bit.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "metal_kernels.npz")
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_metal_golden as G  # noqa: E402

# image relative-L2 bounds, FP64 oracle vs FP32 shader
TOL = {"straight": 2e-5, "curved": 5e-6, "vti": 5e-6}


@pytest.fixture(scope="module")
def fx():
    oracle.build()
    return dict(np.load(FIXTURE))


def _oracle_case(d, spec):
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    name, kind, vel, grid, t0ms, aa, spr, obl, (v0, k), eta = spec
    f64 = lambda a: np.asarray(a, np.float64)
    tb = create_trace_block(d["amps"], f64(d["sx"]), f64(d["sy"]), f64(d["rx"]), f64(d["ry"]),
                            sample_rate_ms=G.DT_MS, start_time_ms=t0ms)
    X, Y = (d["X"], d["Y"]) if grid == "axes" else (d["Xr"], d["Yr"])
    out = OutputTile(image=np.zeros((G.NX, G.NY, G.NT)), fold=np.zeros((G.NX, G.NY), np.int32),
                     x_axis=f64(d["X"][:, 0]), y_axis=f64(d["Y"][0, :]), t_axis_ms=f64(d["t_ms"]),
                     x_grid=None if grid == "axes" else f64(X), y_grid=None if grid == "axes" else f64(Y))
    v = f64(d["v3"] if vel == "3d" else d["v1"])
    kt = {"straight": "straight_ray", "curved": "curved_ray", "vti": "anisotropic_vti"}[kind]
    cfg = KernelConfig(max_aperture_m=G.APERTURE, min_aperture_m=G.APERTURE, max_dip_degrees=45.0,
                       taper_fraction=G.TAPER, aa_enabled=bool(aa), apply_spreading=bool(spr),
                       apply_obliquity=bool(obl), grid_dx=G.DX, grid_dy=G.DX, aa_dominant_freq=30.0,
                       kernel_type=kt, curved_ray_enabled=kind == "curved", curved_ray_v0=v0, curved_ray_k=k,
                       vti_enabled=kind == "vti", vti_eta_array=f64(d["eta1"]) if eta == "1d" else None,
                       vti_eta_constant=eta if isinstance(eta, float) else 0.0)
    oracle.migrate(tb, out, VelocitySlice(vrms=v, is_1d=vel == "1d"), cfg, kind=kt)
    return out


@pytest.mark.parametrize("variant", ["", "_simd"])
@pytest.mark.parametrize("spec", G.CASES, ids=[c[0] for c in G.CASES])
def test_oracle_matches_metal_kernel(spec, variant, fx):
    name, kind = spec[0], spec[1]
    out = _oracle_case(fx, spec)
    ref = fx[f"{name}{variant}_image"].astype(np.float64)
    assert np.abs(ref).max() > 0
    assert rel_l2(out.image, ref) <= TOL[kind]
    if kind != "straight":
        np.testing.assert_array_equal(out.fold, fx[f"{name}{variant}_fold"])
        assert out.fold.min() > 0


def test_oracle_matches_metal_time_variant_kernel(fx):
    """The shader migrates at the window times with v_rms at the base sample at
    or below each time; the windows start on base samples, so that is the
    oracle on the windowed time axis with v_rms taken there."""
    from pstm_b200 import time_variant as tvm
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    f64 = lambda a: np.asarray(a, np.float64)
    tv = tvm.window_times(G.tv_windows())
    assert len(tv) == fx["tv_image"].shape[-1] and np.allclose(tv % G.DT_MS, 0.0)
    v3 = f64(fx["v3"])
    vel = v3[..., np.minimum((tv / G.DT_MS).astype(int), v3.shape[-1] - 1)]
    tb = create_trace_block(fx["amps"], f64(fx["sx"]), f64(fx["sy"]), f64(fx["rx"]), f64(fx["ry"]),
                            sample_rate_ms=G.DT_MS)
    out = OutputTile(image=np.zeros((G.NX, G.NY, len(tv))), fold=np.zeros((G.NX, G.NY), np.int32),
                     x_axis=f64(fx["X"][:, 0]), y_axis=f64(fx["Y"][0, :]), t_axis_ms=tv)
    cfg = KernelConfig(max_aperture_m=G.APERTURE, min_aperture_m=G.APERTURE, max_dip_degrees=45.0,
                       taper_fraction=G.TAPER, aa_enabled=True, grid_dx=G.DX, grid_dy=G.DX, aa_dominant_freq=30.0)
    oracle.migrate(tb, out, VelocitySlice(vrms=vel, is_1d=False), cfg)
    ref = fx["tv_image"].astype(np.float64)
    assert np.abs(ref).max() > 0
    assert rel_l2(out.image, ref) <= TOL["straight"]


def test_traveltime_helpers_match_metal(fx):
    """Two-leg curved-ray and VTI traveltimes: within 2 us of the FP32 shader
    helpers (1e-3 of a 2 ms sample; the shaders' FP32 log of a ratio near 1
    has an absolute, not relative, error at short times)."""
    n = len(fx["h_t0"])
    z = np.zeros(n)
    rows = lambda v, eta: np.stack([fx["h_t0"], fx["h_hs"], z, fx["h_hr"], z, v, eta], 1).astype(np.float64)
    curved = oracle.traveltime("curved_ray", rows(fx["h_v"], fx["h_eta"]), v0=float(fx["h_v0"]),
                               k=float(fx["h_k"]))
    assert np.max(np.abs(curved - fx["h_curved"])) <= 2e-6
    vti = oracle.traveltime("anisotropic_vti", rows(fx["h_v"], fx["h_eta"]))
    assert np.max(np.abs(vti - fx["h_vti"])) <= 2e-6


def test_fixture_is_the_shaders_output():
    from oracle import metal_ref
    if not metal_ref.available():
        pytest.skip("the shader library is built only where the reference tree is")
    d = dict(np.load(FIXTURE))
    for spec in G.CASES:
        for simd, variant in ((False, ""), (True, "_simd")):
            img, fold = G.run_case(metal_ref, d, spec, simd=simd)
            np.testing.assert_array_equal(img, d[f"{spec[0]}{variant}_image"])
            np.testing.assert_array_equal(fold, d[f"{spec[0]}{variant}_fold"])
    img, fold = G.run_tv(metal_ref, d)
    np.testing.assert_array_equal(img, d["tv_image"])
    np.testing.assert_array_equal(fold, d["tv_fold"])
    h = G.helper_rows(metal_ref)
    for key, val in h.items():
        np.testing.assert_array_equal(val, d[key])
