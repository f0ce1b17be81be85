"""Test infrastructure only: the FP64 CPU restatement of the warm-start network.

The B200 library's learned warm start (xhdfe-xfe_b200/csrc/mlp_kernels.cuh,
xhdfe-xfe_b200/learned.py) is a 3-hidden-layer, 64-wide MLP with BF16 weights and
activations and FP32 accumulation.  It has no counterpart in the reference; this
module is the CPU oracle its device forward pass and gradients are checked
against (tests/test_mlp.py, tests/test_gpu_learned.py):

    x  (8 features, rounded to BF16)
    h1 = bf16(relu(W1 x  + b1))      W1: 64 x 8
    h2 = bf16(relu(W2 h1 + b2))      W2: 64 x 64
    h3 = bf16(relu(W3 h2 + b3))      W3: 64 x 64
    y  = W4 h3 + b4                  W4: 2 x 64      (y: warm-start correction,
                                                      log diagonal scaling)

Weights are the BF16 roundings of FP32 master parameters, biases stay FP32.
Loss: L = (1/N) sum_s sum_o w_so (y_so - t_so)^2.  Gradients are those of L
with respect to the master parameters, the BF16 roundings taken as identity
(straight-through), and the ReLU derivative taken as [h > 0] on the rounded
activation; computed here in FP64 from the same rounded values the device
uses, so the device gradient differs only by its FP32 accumulation.

Flat parameter layout (FP32, 9026 values): W1 (64x8, row-major), b1 (64),
W2 (64x64), b2 (64), W3 (64x64), b3 (64), W4 (2x64), b4 (2).
"""

from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 8, 64, 2
SHAPES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
          ("W3", (N_HID, N_HID)), ("b3", (N_HID,)), ("W4", (N_OUT, N_HID)), ("b4", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    bits = f.view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    out = rounded.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    if nan.any():
        out[nan] = np.nan
    return out


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases, a zero output layer (the untrained
    network predicts no correction)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        if name.startswith("b") or name == "W4":
            parts.append(np.zeros(shape))
        else:
            lim = np.sqrt(6.0 / shape[1])
            parts.append(rng.uniform(-lim, lim, shape))
    return np.concatenate([x.ravel() for x in parts]).astype(np.float32)


def forward(params, X, rounding: bool = True):
    """Outputs (N x 2) and the cached values of the backward pass.  With
    rounding=False every BF16/FP32 rounding is skipped (exact FP64 network, for
    finite-difference checks of the backward formulas)."""
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    P = unpack(params)
    W = {k: rnd(v) if k.startswith("W") else
         (np.asarray(v, dtype=np.float32).astype(np.float64) if rounding else np.asarray(v, dtype=np.float64))
         for k, v in P.items()}
    x = rnd(X)
    z1 = x @ W["W1"].T + W["b1"]
    h1 = rnd(np.maximum(z1, 0.0))
    z2 = h1 @ W["W2"].T + W["b2"]
    h2 = rnd(np.maximum(z2, 0.0))
    z3 = h2 @ W["W3"].T + W["b3"]
    h3 = rnd(np.maximum(z3, 0.0))
    y = h3 @ W["W4"].T + W["b4"]
    return y, (W, x, z1, h1, z2, h2, z3, h3)


def loss_and_grad(params, X, T, rounding: bool = True):
    """Loss and gradient (flat, FP64) for targets T = [t0, t1, w0, w1] per row."""
    T = np.asarray(T, dtype=np.float64)
    n = X.shape[0]
    y, (W, x, z1, h1, z2, h2, z3, h3) = forward(params, X, rounding)
    t, w = T[:, :2], T[:, 2:4]
    diff = y - t
    loss = float((w * diff * diff).sum() / n)
    dy = 2.0 * w * diff / n
    g = {}
    g["W4"] = dy.T @ h3
    g["b4"] = dy.sum(0)
    d3 = (dy @ W["W4"]) * (h3 > 0)
    g["W3"] = d3.T @ h2
    g["b3"] = d3.sum(0)
    d2 = (d3 @ W["W3"]) * (h2 > 0)
    g["W2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ W["W2"]) * (h1 > 0)
    g["W1"] = d1.T @ x
    g["b1"] = d1.sum(0)
    flat = np.concatenate([g[name].ravel() for name, _ in SHAPES])
    return loss, flat


def adam_step(params, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba, 2015) of FP32 master parameters, in FP64."""
    m = beta1 * m + (1.0 - beta1) * grad
    v = beta2 * v + (1.0 - beta2) * grad * grad
    mh = m / (1.0 - beta1 ** step)
    vh = v / (1.0 - beta2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
