"""The CUDA path against the reference's own Metal shader kernels (GPU).

``tests/golden/metal_kernels.npz`` holds the outputs of the reference's
pstm_migrate_3d, pstm_migrate_curved_ray and pstm_migrate_vti shaders
(compiled as C++ and run on the CPU by ``tests/golden/make_metal_golden.py``)
on FP32-exact inputs with a constant aperture.  The CUDA backend, through
its public methods on host arrays, must reproduce their images within the
tolerances of the same kinds against the FP64 oracle (1e-5 for every kind on
the FP64 sample-index path, 1e-4 curved and VTI with FP32 traveltime), and the
curved and VTI kernels' (nx, ny) fold exactly.  The time-variant shader's
image at the window times is reproduced by ``migrate_tile_time_variant``."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_metal_golden as G  # noqa: E402

FIXTURE = os.path.join(HERE, "golden", "metal_kernels.npz")

TOL = {"exact": {"straight": 1e-5, "curved": 1e-5, "vti": 1e-5},
       "fast": {"straight": 1e-4, "curved": 1e-4, "vti": 1e-4}}


@pytest.mark.parametrize("precision", ["exact", "fast"])
@pytest.mark.parametrize("spec", G.CASES, ids=[c[0] for c in G.CASES])
def test_cuda_matches_metal_kernel(spec, precision, cuda_kernel_factory):
    import dataclasses
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    d = dict(np.load(FIXTURE))
    name, kind, vel, grid, t0ms, aa, spr, obl, (v0, k), eta = spec
    f64 = lambda a: np.asarray(a, np.float64)
    tb = create_trace_block(d["amps"], f64(d["sx"]), f64(d["sy"]), f64(d["rx"]), f64(d["ry"]),
                            sample_rate_ms=G.DT_MS, start_time_ms=t0ms)
    X, Y = (d["X"], d["Y"]) if grid == "axes" else (d["Xr"], d["Yr"])
    out = OutputTile(image=np.zeros((G.NX, G.NY, G.NT)), fold=np.zeros((G.NX, G.NY), np.int32),
                     x_axis=f64(d["X"][:, 0]), y_axis=f64(d["Y"][0, :]), t_axis_ms=f64(d["t_ms"]),
                     x_grid=None if grid == "axes" else f64(X), y_grid=None if grid == "axes" else f64(Y))
    kt = {"straight": "straight_ray", "curved": "curved_ray", "vti": "anisotropic_vti"}[kind]
    cfg = KernelConfig(max_aperture_m=G.APERTURE, min_aperture_m=G.APERTURE, max_dip_degrees=45.0,
                       taper_fraction=G.TAPER, aa_enabled=bool(aa), apply_spreading=bool(spr),
                       apply_obliquity=bool(obl), grid_dx=G.DX, grid_dy=G.DX, aa_dominant_freq=30.0,
                       kernel_type=kt, curved_ray_enabled=kind == "curved", curved_ray_v0=v0, curved_ray_k=k,
                       vti_enabled=kind == "vti", vti_eta_array=f64(d["eta1"]) if eta == "1d" else None,
                       vti_eta_constant=eta if isinstance(eta, float) else 0.0)
    kern = cuda_kernel_factory(cfg, precision=precision)
    method = {"straight": kern.migrate_tile, "curved": kern.migrate_tile_curved_ray,
              "vti": kern.migrate_tile_vti}[kind]
    method(tb, out, VelocitySlice(vrms=f64(d["v3"] if vel == "3d" else d["v1"]), is_1d=vel == "1d"), cfg)
    ref = d[f"{name}_image"].astype(np.float64)
    assert rel_l2(out.image, ref) <= TOL[precision][kind]
    if kind != "straight":
        np.testing.assert_array_equal(out.fold, d[f"{name}_fold"])


def test_cuda_time_variant_matches_metal_kernel(cuda_kernel_factory):
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    d = dict(np.load(FIXTURE))
    f64 = lambda a: np.asarray(a, np.float64)
    tb = create_trace_block(d["amps"], f64(d["sx"]), f64(d["sy"]), f64(d["rx"]), f64(d["ry"]),
                            sample_rate_ms=G.DT_MS)
    out = OutputTile(image=np.zeros((G.NX, G.NY, G.NT)), fold=np.zeros((G.NX, G.NY), np.int32),
                     x_axis=f64(d["X"][:, 0]), y_axis=f64(d["Y"][0, :]), t_axis_ms=f64(d["t_ms"]))
    cfg = KernelConfig(max_aperture_m=G.APERTURE, min_aperture_m=G.APERTURE, max_dip_degrees=45.0,
                       taper_fraction=G.TAPER, aa_enabled=True, grid_dx=G.DX, grid_dy=G.DX, aa_dominant_freq=30.0)
    kern = cuda_kernel_factory(cfg)
    kern.migrate_tile_time_variant(tb, out, VelocitySlice(vrms=f64(d["v3"]), is_1d=False), cfg, G.tv_windows())
    ref = d["tv_image"].astype(np.float64)
    assert out.image.shape == ref.shape
    assert rel_l2(out.image, ref) <= TOL["exact"]["straight"]
