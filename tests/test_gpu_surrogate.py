"""The learned traveltime form on the GPU.

* exact training targets of the sample kernel vs the FP64 oracle (1e-12);
* gradients of the tensor-core forward/backward kernel vs the NumPy oracle that
  rounds to BF16 at the same points (relative L2 <= 2e-2 per parameter block;
  the kernel's SiLU uses the hardware tanh);
* training with the package's own kernels lowers the loss;
* the learned migration kernel: with eta = 0 and a network whose output is 0
  the surrogate time is the straight DSR time, which is the exact VTI time, so
  the learned kernel must reproduce the exact kernel (relative L2 <= 1e-4,
  fold bit-exact);
* ablation: a network that ignores the VTI term fails the 0.1 ms probe and the
  tile falls back to the exact kernel (bit-identical image); forcing it changes
  the image.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle
from oracle import surrogate_ref as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trainer():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pstm_b200 import build
    build.build()
    from pstm_b200 import surrogate as S
    t = S.Trainer(0)
    yield t
    t.close()


@pytest.mark.parametrize("kind", ["anisotropic_vti", "curved_vti"])
def test_sample_targets_match_oracle(trainer, kind):
    from pstm_b200 import surrogate as S
    dom = S.survey_domain(kind, h_max_m=3200.0, v0=1600.0, k=0.4)
    raw, res, tex = trainer.samples(dom, 99, 1000, 2048, with_exact=True)
    f = raw[:, :7].double().cpu().numpy()
    ref = oracle.traveltime(kind, f, v0=1600.0, k=0.4)
    np.testing.assert_allclose(tex.cpu().numpy(), ref, rtol=1e-12, atol=1e-12)
    dsr = oracle.traveltime("straight_ray", f)
    np.testing.assert_allclose(res.double().cpu().numpy(), ref - dsr, rtol=1e-6, atol=1e-7)


def test_gradients_match_oracle(trainer):
    import torch
    from pstm_b200 import surrogate as S
    dom = S.survey_domain("anisotropic_vti", h_max_m=3200.0)
    raw, res, _ = trainer.samples(dom, 5, 0, 300)   # not a multiple of the 128-sample CTA
    p = S.init_params(3)
    p[-1] = 0.1
    net = S.Net(torch.as_tensor(p, device="cuda"), dom, out_scale=0.5)
    g, loss = trainer.gradients(net, raw, res)
    shift, scale = dom.norm()
    xn = (raw[:, :7].double().cpu().numpy() - np.array(shift[:7])) * np.array(scale[:7])
    xn = xn.astype(np.float32).astype(np.float64)   # the kernel normalises in FP32
    tgt = res.double().cpu().numpy() / 0.5
    loss_ref, g_ref, _ = R.forward_backward(p.astype(np.float64), xn, tgt, bf16_points=True)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    gk = g.double().cpu().numpy()
    o = 0
    for name, shape in R.SHAPES:
        n = int(np.prod(shape))
        a, b = gk[o:o + n], g_ref[o:o + n]
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-9, name
        o += n


def test_training_lowers_the_loss(trainer):
    from pstm_b200 import surrogate as S
    dom = S.survey_domain("anisotropic_vti", h_max_m=3200.0)
    net = trainer.train(dom, n_train=1 << 22, steps=400, batch=8192, lr=3e-3, log_every=100)
    losses = [h[1] for h in net.history]
    assert losses[-1] < 0.3 * losses[0], losses
    err = trainer.error_ms(net, n=1 << 16)
    assert np.isfinite(err["max_ms"]) and err["rms_ms"] > 0


def _tile(n_traces=1500, nx=6, ny=5, nt=300, eta_zero=False):
    import torch
    from pstm_b200 import workloads
    from pstm_b200.base import OutputTile, TraceBlock, VelocitySlice
    case = workloads.config2_small(n_traces=n_traces, nx=nx, ny=ny, nt=nt, ns=nt)
    tb, out = case.traces, case.output
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    dtb = TraceBlock(amplitudes=dev(tb.amplitudes), source_x=dev(tb.source_x), source_y=dev(tb.source_y),
                     receiver_x=dev(tb.receiver_x), receiver_y=dev(tb.receiver_y), offset=dev(tb.offset),
                     midpoint_x=dev(tb.midpoint_x), midpoint_y=dev(tb.midpoint_y),
                     sample_rate_ms=tb.sample_rate_ms, start_time_ms=tb.start_time_ms)
    eta = np.zeros(nt) if eta_zero else workloads.survey_eta(out.t_axis_ms)
    cfg = workloads.survey_config(kernel_type="anisotropic_vti", aa=True, eta=eta)
    cfg.vti_eta_array = dev(eta)

    def fresh():
        return OutputTile(image=torch.zeros(out.image.shape, dtype=torch.float64, device="cuda"),
                          fold=torch.zeros(out.fold.shape, dtype=torch.int32, device="cuda"),
                          x_axis=dev(out.x_axis), y_axis=dev(out.y_axis), t_axis_ms=dev(out.t_axis_ms))
    return dtb, fresh, VelocitySlice(vrms=dev(case.velocity.vrms), is_1d=False), cfg


def test_learned_kernel_reproduces_exact_when_the_surrogate_is_exact(cuda_kernel_factory):
    import torch
    from pstm_b200 import surrogate as S
    dtb, fresh, vel, cfg = _tile(eta_zero=True)
    k = cuda_kernel_factory(cfg)
    ref = fresh()
    k.migrate_tile_vti(dtb, ref, vel, cfg)
    zero = S.Net(torch.zeros(S.N_PARAMS, dtype=torch.float32, device="cuda"),
                 S.survey_domain("anisotropic_vti", h_max_m=3200.0), out_scale=0.5)
    got = fresh()
    _, rep = k.migrate_tile_learned(dtb, got, vel, zero, cfg, max_residual_ms=-1.0)
    torch.cuda.synchronize()
    assert rep["used_surrogate"] and rep["n_probe_used"] > 0
    assert rep["probe_max_ms"] < 1e-2   # T_DSR in FP32 vs the exact FP64 time
    np.testing.assert_array_equal(got.fold.cpu().numpy(), ref.fold.cpu().numpy())
    assert rel_l2(got.image.cpu().numpy(), ref.image.cpu().numpy()) <= 1e-4


def test_ablation_probe_falls_back_to_exact(cuda_kernel_factory):
    import torch
    from pstm_b200 import surrogate as S
    dtb, fresh, vel, cfg = _tile()
    k = cuda_kernel_factory(cfg)
    ref = fresh()
    k.migrate_tile_vti(dtb, ref, vel, cfg)
    blind = S.Net(torch.zeros(S.N_PARAMS, dtype=torch.float32, device="cuda"),
                  S.survey_domain("anisotropic_vti", h_max_m=3200.0), out_scale=0.5)   # no VTI term
    got = fresh()
    _, rep = k.migrate_tile_learned(dtb, got, vel, blind, cfg, max_residual_ms=0.1)
    torch.cuda.synchronize()
    assert not rep["used_surrogate"] and rep["probe_max_ms"] > 0.1
    np.testing.assert_array_equal(got.image.cpu().numpy(), ref.image.cpu().numpy())
    np.testing.assert_array_equal(got.fold.cpu().numpy(), ref.fold.cpu().numpy())
    forced = fresh()
    _, rep2 = k.migrate_tile_learned(dtb, forced, vel, blind, cfg, max_residual_ms=-1.0)
    torch.cuda.synchronize()
    assert rep2["used_surrogate"]
    assert rel_l2(forced.image.cpu().numpy(), ref.image.cpu().numpy()) > 1e-3
    with pytest.raises(ValueError, match="another traveltime kind"):
        cv = S.Net(blind.params, S.survey_domain("curved_vti"), out_scale=0.5)
        k.migrate_tile_learned(dtb, fresh(), vel, cv, cfg)
