"""The FP64 oracle against the reference's own outputs (CPU only)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_files, interp_velocity, load_golden_case, rel_l2
from oracle import oracle


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: os.path.basename(p)[6:-4])
def test_oracle_matches_reference_numba(path):
    tb, out, vel, cfg, img_ref, fold_ref = load_golden_case(path)
    oracle.migrate(tb, out, interp_velocity(vel, out.t_axis_ms), cfg, kind="straight_ray")
    np.testing.assert_array_equal(out.fold, fold_ref)
    if np.abs(img_ref).max() == 0:
        assert np.abs(out.image).max() == 0
    else:
        assert rel_l2(out.image, img_ref) < 1e-12


def test_oracle_accumulates_in_place():
    """image += and fold += like numba_cpu_optimized.py:225-231."""
    tb, out, vel, cfg, img_ref, fold_ref = load_golden_case(os.path.join(GOLDEN, "numba_weights_taper.npz"))
    v = interp_velocity(vel, out.t_axis_ms)
    oracle.migrate(tb, out, v, cfg)
    oracle.migrate(tb, out, v, cfg)
    np.testing.assert_array_equal(out.fold, 2 * fold_ref)
    assert rel_l2(out.image, 2 * img_ref) < 1e-12


def test_oracle_pillar_subset_equals_full():
    tb, out, vel, cfg, img_ref, fold_ref = load_golden_case(os.path.join(GOLDEN, "numba_c1_subset.npz"))
    v = interp_velocity(vel, out.t_axis_ms)
    ny = out.image.shape[1]
    oracle.migrate(tb, out, v, cfg, pillars=(3 * ny, 5 * ny))
    np.testing.assert_array_equal(out.fold[3:5], fold_ref[3:5])
    assert np.all(out.fold[:3] == 0) and np.all(out.fold[5:] == 0)
    assert rel_l2(out.image[3:5], img_ref[3:5]) < 1e-12


def test_oracle_traveltimes_match_reference_python():
    z = np.load(os.path.join(GOLDEN, "traveltime_curved_vti.npz"))
    m = len(z["t0"])
    feat = np.zeros((m, 7))
    feat[:, 0] = z["t0"]
    feat[:, 1] = z["hs"]   # leg distances along x only: h = |dx|
    feat[:, 3] = z["hr"]
    feat[:, 5] = z["v"]
    feat[:, 6] = z["eta"]
    Tv = oracle.traveltime("anisotropic_vti", feat)
    np.testing.assert_allclose(Tv, z["T_vti"], rtol=1e-13, atol=1e-15)
    Tc = np.array([oracle.traveltime("curved_ray", feat[i:i + 1], z["v0"][i], z["k"][i])[0] for i in range(m)])
    np.testing.assert_allclose(Tc, z["T_curved"], rtol=1e-12, atol=1e-14)


def test_oracle_linear_interp_known_answers():
    """Known answers of the reference's tests/test_interpolation.py:88-100."""
    assert oracle.linear_interp([0.0, 1.0, 2.0, 3.0, 4.0], 2.0) == 2.0
    assert oracle.linear_interp([0.0, 2.0, 4.0], 0.5) == 1.0
    assert oracle.linear_interp([0.0, 1.0, 2.0], -1.0) == 0.0
    assert oracle.linear_interp([0.0, 1.0, 2.0], 5.0) == 0.0


def test_oracle_straight_is_curved_with_zero_gradient():
    """curved_ray.py:35-38: |k| < 1e-10 is straight rays at v0."""
    rng = np.random.default_rng(0)
    feat = np.column_stack([rng.uniform(0.01, 3, 50), rng.uniform(-2000, 2000, (50, 4)),
                            np.full(50, 1800.0), np.zeros(50)])
    np.testing.assert_allclose(oracle.traveltime("curved_ray", feat, 1800.0, 0.0),
                               oracle.traveltime("straight_ray", feat), rtol=1e-14)


def test_oracle_vti_with_zero_eta_is_straight():
    rng = np.random.default_rng(1)
    feat = np.column_stack([rng.uniform(0.01, 3, 50), rng.uniform(-2000, 2000, (50, 4)),
                            rng.uniform(1500, 4000, 50), np.zeros(50)])
    np.testing.assert_allclose(oracle.traveltime("anisotropic_vti", feat),
                               oracle.traveltime("straight_ray", feat), rtol=1e-13)


def test_oracle_rejects_bad_arguments():
    from pstm_b200 import workloads
    case = workloads.config1(n_traces=8, nx=2, ny=2, nt=4)
    case.traces.amplitudes = case.traces.amplitudes[:, :1]   # fewer than 2 samples
    with pytest.raises(ValueError):
        oracle.migrate(case.traces, case.output, case.velocity, case.config)


def test_oracle_interpolators_match_reference_golden():
    """Every trace interpolator of the oracle against the reference's own
    interpolate_sample (tests/golden/interp_methods.npz)."""
    z = np.load(os.path.join(GOLDEN, "interp_methods.npz"))
    codes = dict(zip(z["method_names"], z["reference_codes"]))
    for name in z["method_names"]:
        for i, tr in enumerate(z["traces"]):
            for j, t in enumerate(z["t_samples"]):
                got = oracle.interp(tr, t, str(name))
                assert abs(got - z["values"][codes[name], i, j]) <= 1e-12, (name, i, t)
