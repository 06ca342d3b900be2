"""The learned traveltime form: training and use of the surrogate network.

The network (``csrc/mlp.cuh``) maps (t0, dx_s, dy_s, dx_r, dy_r, v_rms, eta)
to the difference between the exact VTI (or curved+VTI) traveltime and the
straight-ray DSR time; T = T_DSR + out_scale * net(normalised inputs).  It is
trained here on seeded samples whose exact FP64 targets a CUDA kernel
generates, with this package's own forward/backward and Adam kernels (no
autograd), and used through ``CudaKernel.migrate_tile_learned``, which probes
the network against the exact formula on every tile and falls back to the
exact kernel when the largest residual exceeds the threshold (0.1 ms).

Torch is used only to hold device buffers.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat

N_PARAMS = 8897
KINDS = {"anisotropic_vti": nat.TT_VTI, "curved_vti": nat.TT_CURVED_VTI}


@dataclass
class Domain:
    """Sampling box of the training inputs (the ranges a survey produces)."""
    kind: int = nat.TT_VTI
    t0_max_s: float = 3.0
    h_max_m: float = 4500.0
    v_a: float = 1500.0            # v_rms = (v_a + v_b t0)(1 + v_rel u)
    v_b: float = 2500.0 / 3.0
    v_rel: float = 0.2
    eta_slope: float = 0.05        # eta = clip(eta_slope t0 + eta_jitter u', 0, eta_max)
    eta_jitter: float = 0.03
    eta_max: float = 0.15
    curved_v0: float = 1500.0
    curved_k: float = 0.5

    def to_struct(self) -> nat.SurrogateDomain:
        d = nat.SurrogateDomain()
        d.traveltime = self.kind
        d.curved_v0, d.curved_k = self.curved_v0, self.curved_k
        d.t0_max_s, d.h_max_m = self.t0_max_s, self.h_max_m
        d.v_a, d.v_b, d.v_rel = self.v_a, self.v_b, self.v_rel
        d.eta_slope, d.eta_jitter, d.eta_max = self.eta_slope, self.eta_jitter, self.eta_max
        return d

    def norm(self):
        """(shift, scale) mapping every input range onto about [-1, 1]."""
        v_lo = self.v_a * (1.0 - self.v_rel)
        v_hi = (self.v_a + self.v_b * self.t0_max_s) * (1.0 + self.v_rel)
        lo = [0.0, -self.h_max_m, -self.h_max_m, -self.h_max_m, -self.h_max_m, v_lo, 0.0, 0.0]
        hi = [self.t0_max_s, self.h_max_m, self.h_max_m, self.h_max_m, self.h_max_m, v_hi,
              max(self.eta_max, 1e-6), 1.0]
        shift = [(a + b) / 2.0 for a, b in zip(lo, hi)]
        scale = [2.0 / (b - a) for a, b in zip(lo, hi)]
        return shift, scale


def survey_domain(kind: str = "anisotropic_vti", t0_max_s: float = 3.0, h_max_m: float = 4500.0,
                  v0: float = 1500.0, k: float = 0.5) -> Domain:
    """The ranges of the survey cases: v_rms = (1500 + 2500 t/3 s)(1 + 0.05 G),
    |G| < 4, eta(t0) = 0.15 t0 / 3 s, output-point-to-source/receiver
    distances up to h_max_m per axis."""
    return Domain(kind=KINDS[kind], t0_max_s=t0_max_s, h_max_m=h_max_m, v_rel=0.2, eta_slope=0.05,
                  eta_jitter=0.03, eta_max=0.15, curved_v0=v0, curved_k=k)


@dataclass
class Net:
    params: object                 # torch float32 CUDA tensor (N_PARAMS,)
    domain: Domain
    out_scale: float
    history: list = field(default_factory=list)

    def to_struct(self) -> nat.Surrogate:
        s = nat.Surrogate()
        shift, scale = self.domain.norm()
        for i in range(8):
            s.shift[i] = shift[i]
            s.scale[i] = scale[i]
        s.out_scale = self.out_scale
        s.traveltime = self.domain.kind
        s.params = self.params.data_ptr()
        return s

    def save(self, path: str) -> None:
        d = self.domain
        np.savez(path, params=self.params.detach().cpu().numpy(), out_scale=self.out_scale,
                 domain=np.array([d.kind, d.t0_max_s, d.h_max_m, d.v_a, d.v_b, d.v_rel, d.eta_slope,
                                  d.eta_jitter, d.eta_max, d.curved_v0, d.curved_k]))

    @staticmethod
    def load(path: str, device="cuda") -> "Net":
        import torch
        z = np.load(path)
        v = z["domain"]
        dom = Domain(kind=int(v[0]), t0_max_s=v[1], h_max_m=v[2], v_a=v[3], v_b=v[4], v_rel=v[5],
                     eta_slope=v[6], eta_jitter=v[7], eta_max=v[8], curved_v0=v[9], curved_k=v[10])
        return Net(torch.as_tensor(z["params"], device=device), dom, float(z["out_scale"]))


def init_params(seed: int) -> np.ndarray:
    """Flat FP32 parameters: weights uniform in +-sqrt(6 / (fan_in + fan_out)),
    biases zero (layout W1[64][7] b1 W2[64][64] b2 W3 b3 w4[64] b4)."""
    rng = np.random.default_rng(seed)
    parts = []
    for shape, fan in (((64, 7), (7, 64)), ((64,), None), ((64, 64), (64, 64)), ((64,), None),
                       ((64, 64), (64, 64)), ((64,), None), ((64,), (64, 1)), ((1,), None)):
        if fan is None:
            parts.append(np.zeros(shape))
        else:
            lim = math.sqrt(6.0 / (fan[0] + fan[1]))
            parts.append(rng.uniform(-lim, lim, shape))
    flat = np.concatenate([p.ravel() for p in parts]).astype(np.float32)
    assert flat.size == N_PARAMS
    return flat


class Trainer:
    """Own-kernel training of the surrogate on one CUDA device."""

    def __init__(self, device: int = 0):
        import torch
        self.L = nat.load()
        if self.L.pstm_cuda_surrogate_param_count() != N_PARAMS:
            raise RuntimeError("surrogate parameter count mismatch; rebuild libpstm_cuda.so")
        self.device = device
        h = ctypes.c_void_p()
        nat.check(self.L.pstm_cuda_create(device, ctypes.byref(h)), None, self.L)
        self.ctx = h
        self.torch = torch

    def close(self):
        if self.ctx is not None:
            self.L.pstm_cuda_destroy(self.ctx)
            self.ctx = None

    def _stream(self):
        return self.torch.cuda.current_stream().cuda_stream or nat.STREAM_LEGACY

    def samples(self, domain: Domain, seed: int, first: int, n: int, with_exact: bool = False):
        """(raw (n, 8) float32, residual (n,) float32 [s], exact T (n,) float64 or None)."""
        torch = self.torch
        raw = torch.empty((n, 8), dtype=torch.float32, device="cuda")
        res = torch.empty((n,), dtype=torch.float32, device="cuda")
        tex = torch.empty((n,), dtype=torch.float64, device="cuda") if with_exact else None
        dom = domain.to_struct()
        nat.check(self.L.pstm_cuda_surrogate_samples(self.ctx, ctypes.byref(dom), seed & (2**64 - 1), first, n,
                                                     raw.data_ptr(), res.data_ptr(),
                                                     tex.data_ptr() if tex is not None else None,
                                                     ctypes.c_void_p(self._stream())), self.ctx, self.L)
        return raw, res, tex

    def gradients(self, net: Net, raw, residual):
        """(grads (N_PARAMS,) float32 tensor, loss_sum float) of one batch."""
        torch = self.torch
        g = torch.zeros(N_PARAMS, dtype=torch.float32, device="cuda")
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        s = net.to_struct()
        nat.check(self.L.pstm_cuda_surrogate_gradients(self.ctx, ctypes.byref(s), raw.data_ptr(), residual.data_ptr(),
                                                       raw.shape[0], g.data_ptr(), loss.data_ptr(),
                                                       ctypes.c_void_p(self._stream())), self.ctx, self.L)
        return g, float(loss.item())

    def evaluate(self, net: Net, raw):
        """Network residual (s) of the samples."""
        torch = self.torch
        out = torch.empty((raw.shape[0],), dtype=torch.float32, device="cuda")
        s = net.to_struct()
        nat.check(self.L.pstm_cuda_surrogate_eval(self.ctx, ctypes.byref(s), raw.data_ptr(), raw.shape[0],
                                                  out.data_ptr(), ctypes.c_void_p(self._stream())), self.ctx, self.L)
        return out

    def error_ms(self, net: Net, n: int = 1 << 20, seed: int = 987654321) -> dict:
        """Traveltime error of the surrogate on n held-out samples (another
        seed), in ms: |(T_DSR + net) - T_exact| with T_DSR in FP64."""
        raw, res, _ = self.samples(net.domain, seed, 0, n)
        pred = self.evaluate(net, raw)
        err = (pred.double() - res.double()).abs() * 1000.0
        return {"max_ms": float(err.max()), "rms_ms": float(err.pow(2).mean().sqrt()),
                "p99_ms": float(err.float().quantile(0.99)) if n <= (1 << 24) else None, "n": n}

    def train(self, domain: Domain, n_train: int = 50_000_000, steps: int = 6000, batch: int = 65536,
              lr: float = 2e-3, lr_min: float = 1e-5, seed: int = 12345, init_seed: int = 7,
              log_every: int = 500) -> Net:
        """Adam with cosine decay on batches drawn in turn from the n_train
        seeded samples (regenerated on the device, not stored)."""
        torch = self.torch
        params = torch.as_tensor(init_params(init_seed), device="cuda")
        raw, res, _ = self.samples(domain, seed, 0, 1 << 18)
        out_scale = float(res.abs().max()) * 1.05 or 1.0
        net = Net(params, domain, out_scale)
        g = torch.zeros(N_PARAMS, dtype=torch.float32, device="cuda")
        m = torch.zeros_like(g)
        v = torch.zeros_like(g)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        s = net.to_struct()
        st = ctypes.c_void_p(self._stream())
        dom = domain.to_struct()
        raw = torch.empty((batch, 8), dtype=torch.float32, device="cuda")
        res = torch.empty((batch,), dtype=torch.float32, device="cuda")
        t0 = time.perf_counter()
        for step in range(1, steps + 1):
            first = ((step - 1) * batch) % max(batch, n_train - batch)
            nat.check(self.L.pstm_cuda_surrogate_samples(self.ctx, ctypes.byref(dom), seed, first, batch,
                                                         raw.data_ptr(), res.data_ptr(), None, st), self.ctx, self.L)
            nat.check(self.L.pstm_cuda_surrogate_gradients(self.ctx, ctypes.byref(s), raw.data_ptr(), res.data_ptr(),
                                                           batch, g.data_ptr(), loss.data_ptr(), st),
                      self.ctx, self.L)
            lr_t = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * (step - 1) / steps))
            nat.check(self.L.pstm_cuda_surrogate_adam(self.ctx, params.data_ptr(), g.data_ptr(), m.data_ptr(),
                                                      v.data_ptr(), step, lr_t, st), self.ctx, self.L)
            if step % log_every == 0 or step == steps:
                net.history.append((step, float(loss.item()) / (log_every * batch), time.perf_counter() - t0))
                loss.zero_()
        torch.cuda.synchronize()
        return net
