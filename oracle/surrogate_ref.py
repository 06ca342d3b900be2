"""CPU oracle of the traveltime surrogate network (test infrastructure).

A NumPy restatement of the network the CUDA kernels train and evaluate
(7 -> 64 -> 64 -> 64 -> 1, SiLU): forward pass, mean-squared loss on the
normalised residual, and the analytic backward pass.  With ``bf16=True`` it
rounds to BF16 exactly where the tensor-core kernels do (weights, the inputs
of every matrix product, the stored activations and the back-propagated
pre-activation gradients) and keeps everything else in FP64, so the CUDA
gradients can be compared with it; with ``bf16=False`` it is plain FP64, which
the finite-difference test uses.  The reference project has no surrogate
(its traveltimes are closed formulas only), so nothing here follows a
reference file: this oracle checks this repository's own kernels.
"""
from __future__ import annotations

import numpy as np

N_IN, H = 7, 64
SHAPES = [("W1", (H, N_IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
          ("w4", (H,)), ("b4", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)   # 8897


def unpack(flat: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward_backward(flat: np.ndarray, xn: np.ndarray, target: np.ndarray, bf16_points: bool = True):
    """(loss_sum, grads (flat), y) for normalised inputs xn (n, 7) and
    normalised targets (n,); loss = sum over samples of (y - target)^2, the
    gradient is that of the mean."""
    r = bf16 if bf16_points else (lambda a: np.asarray(a, dtype=np.float64))
    p = unpack(flat)
    n = xn.shape[0]
    W1, W2, W3 = r(p["W1"]), r(p["W2"]), r(p["W3"])
    x = r(xn)
    z1 = x @ W1.T + p["b1"]
    h1 = silu(z1)
    z2 = r(h1) @ W2.T + p["b2"]
    h2 = silu(z2)
    z3 = r(h2) @ W3.T + p["b3"]
    h3 = silu(z3)
    y = h3 @ p["w4"] + p["b4"][0]
    e = y - target
    dy = 2.0 * e / n
    g = {"w4": dy @ h3, "b4": np.array([dy.sum()])}
    dz3 = (dy[:, None] * p["w4"][None, :]) * dsilu(z3)
    g["b3"] = dz3.sum(0)
    g["W3"] = r(dz3).T @ r(h2)
    dz2 = (r(dz3) @ W3) * dsilu(z2)
    g["b2"] = dz2.sum(0)
    g["W2"] = r(dz2).T @ r(h1)
    dz1 = (r(dz2) @ W2) * dsilu(z1)
    g["b1"] = dz1.sum(0)
    g["W1"] = r(dz1).T @ x
    return float((e * e).sum()), pack(g), y
