"""Randomised configurations of every traveltime kind, CUDA against the FP64
oracle (GPU).

Each seeded draw picks the kind (straight, curved, VTI, curved+VTI), maximum
and minimum aperture, dip, taper (0 included), spreading and obliquity, AA,
trace weights or none, sample rate and start time, 1-D or 3-D velocity, eta
as a constant or a function of t0, the curved-ray gradient (0 included) and a
2-D or 3-D fold; traces are band-limited noise.  On the FP64 sample-index path
("exact") the image must be within 1e-5 relative L2 of the oracle and the fold
identical; with FP32 traveltime ("fast", and "fp32" whose trace-end tests are
FP32 too) within 1e-4 (on noise-like traces FP32 traveltime alone leaves
~1.1e-5, even for straight rays)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle

pytestmark = pytest.mark.gpu

KINDS = ["straight_ray", "curved_ray", "anisotropic_vti", "curved_vti"]


def _draw(seed):
    from pstm_b200.base import KernelConfig, OutputTile, VelocitySlice, create_trace_block
    rng = np.random.default_rng(1000 + seed)
    kind = KINDS[seed % 4]
    n, ns, nt, nx, ny = 900, 400, 160, 5, 4
    s, r = rng.uniform(0, 2000, (n, 2)), rng.uniform(0, 2000, (n, 2))
    tw = np.arange(-25, 26) * 0.004
    ricker = (1 - 2 * (np.pi * 25 * tw) ** 2) * np.exp(-(np.pi * 25 * tw) ** 2)
    amps = np.array([np.convolve(x, ricker, mode="same") for x in rng.standard_normal((n, ns))], np.float32)
    w = rng.uniform(0.5, 1.5, n) if rng.random() < 0.5 else None
    dt, t_start = float(rng.choice([2.0, 4.0])), float(rng.choice([0.0, 8.0, 40.0]))
    tb = create_trace_block(amps, s[:, 0], s[:, 1], r[:, 0], r[:, 1], sample_rate_ms=dt, start_time_ms=t_start,
                            weights=w)
    x, y = rng.uniform(600, 1200) + 25 * np.arange(nx), rng.uniform(600, 1200) + 25 * np.arange(ny)
    t_ms = 6.0 * np.arange(nt)
    v1 = 1600 + 1800 * t_ms / t_ms[-1]
    if rng.random() < 0.5:
        vel = VelocitySlice(vrms=v1, is_1d=True)
    else:
        lat = 1.0 + 0.05 * rng.standard_normal((nx, ny, 1))
        vel = VelocitySlice(vrms=np.ascontiguousarray(v1[None, None, :] * lat), is_1d=False)
    eta_arr = None
    eta_c = 0.0
    if "vti" in kind:
        if rng.random() < 0.5:
            eta_arr = np.clip(0.15 * t_ms / 1000.0 + 0.01 * rng.standard_normal(nt), 0.0, 0.2)
        else:
            eta_c = float(rng.uniform(0.0, 0.2))
    k_grad = float(rng.choice([0.0, rng.uniform(0.2, 1.2)]))
    cfg = KernelConfig(max_aperture_m=float(rng.uniform(400, 2000)), min_aperture_m=float(rng.uniform(50, 400)),
                       max_dip_degrees=float(rng.uniform(20, 80)),
                       taper_fraction=float(rng.choice([0.0, rng.uniform(0.05, 0.4)])),
                       apply_spreading=bool(rng.random() < 0.7), apply_obliquity=bool(rng.random() < 0.7),
                       aa_enabled=bool(rng.random() < 0.6), grid_dx=25.0, grid_dy=25.0, kernel_type=kind,
                       curved_ray_enabled=kind.startswith("curved"), curved_ray_v0=float(rng.uniform(1400, 1800)),
                       curved_ray_k=k_grad, vti_enabled="vti" in kind, vti_eta_array=eta_arr,
                       vti_eta_constant=eta_c)
    fold_shape = (nx, ny) if rng.random() < 0.5 else (nx, ny, nt)
    out = OutputTile(image=np.zeros((nx, ny, nt)), fold=np.zeros(fold_shape, np.int32), x_axis=x, y_axis=y,
                     t_axis_ms=t_ms)
    return kind, tb, out, vel, cfg


@pytest.mark.parametrize("precision", ["exact", "fast", "fp32"])
@pytest.mark.parametrize("seed", range(12))
def test_random_configuration_vs_oracle(seed, precision, cuda_kernel_factory):
    from pstm_b200.base import OutputTile
    kind, tb, out, vel, cfg = _draw(seed)
    k = cuda_kernel_factory(cfg, precision=precision)
    method = {"straight_ray": k.migrate_tile, "curved_ray": k.migrate_tile_curved_ray,
              "anisotropic_vti": k.migrate_tile_vti, "curved_vti": k.migrate_tile_curved_vti}[kind]
    method(tb, out, vel, cfg)
    ref = OutputTile(image=np.zeros_like(out.image), fold=np.zeros_like(out.fold), x_axis=out.x_axis,
                     y_axis=out.y_axis, t_axis_ms=out.t_axis_ms)
    oracle.migrate(tb, ref, vel, cfg, kind=kind)
    np.testing.assert_array_equal(out.fold, ref.fold)
    if np.abs(ref.image).max() == 0:
        assert np.abs(out.image).max() == 0
        return
    tol = 1e-5 if precision == "exact" else 1e-4
    err = rel_l2(out.image, ref.image)
    assert err <= tol, (kind, err)
