"""Learned warm start of the absorber (no counterpart in the reference).

A 3-hidden-layer, 64-wide MLP (BF16 weights and activations, FP32
accumulation; kernels in csrc/mlp_kernels.cuh) maps per-level features of the
Schur system S a = b (its first three Jacobi iterates scaled by the column's
RMS, the level's weight and mobility share, a small-dim flag;
csrc/ws_kernels.cuh) to a correction of the third Jacobi iterate and a
log-scaling of the level's Jacobi diagonal.  It is trained, by this library's
own forward/backward kernels and Adam on the device, on converged solutions
that the plain solver produces (``collect_samples``), and installed in an
``Absorber`` with ``set_warm_start``: every later absorption then starts its
FP64-checked refinement from the prediction.  The plain solver still runs to
the stated tolerance, so only the iteration count changes.

All arrays here are torch CUDA tensors; nothing runs on the CPU.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import _lib
from .absorber import Absorber, make_options, _ptr_array

HERE = Path(__file__).resolve().parent
TRAINED = HERE / "warmstart_mlp.npz"   # parameters trained by train_warmstart.py
N_FEATURES = 8
N_OUT = 2
MODE_START, MODE_SCALE = 1, 2
_SHAPES = [("W1", (64, 8)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)), ("W3", (64, 64)),
           ("b3", (64,)), ("W4", (2, 64)), ("b4", (2,))]


def num_params() -> int:
    return int(_lib.load().b200fe_mlp_num_params())


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform hidden weights, zero biases and a zero output layer, so the
    untrained network predicts no correction (the start is the third Jacobi
    iterate)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in _SHAPES:
        if name.startswith("b") or name == "W4":
            parts.append(np.zeros(shape))
        else:
            lim = np.sqrt(6.0 / shape[1])
            parts.append(rng.uniform(-lim, lim, shape))
    p = np.concatenate([x.ravel() for x in parts]).astype(np.float32)
    assert p.size == num_params()
    return p


def _check(ab: Absorber, rc: int):
    if rc != _lib.OK:
        raise ab._err(rc)


def forward(ab: Absorber, params, x):
    """y (n, 2) = MLP(x (n, 8)); params a float32 CUDA tensor."""
    import torch
    x = x.contiguous()
    y = torch.empty((x.shape[0], N_OUT), dtype=torch.float32, device=x.device)
    _check(ab, ab.lib.b200fe_mlp_forward(ab.handle, params.data_ptr(), x.data_ptr(), x.shape[0],
                                         y.data_ptr()))
    return y


def grad(ab: Absorber, params, x, t):
    """(gradient float64 tensor of num_params, loss) of the weighted squared
    error against targets t (n, 4) = (t0, t1, w0, w1)."""
    import torch
    out = torch.empty(num_params() + 1, dtype=torch.float64, device=x.device)
    _check(ab, ab.lib.b200fe_mlp_grad(ab.handle, params.data_ptr(), x.contiguous().data_ptr(),
                                      t.contiguous().data_ptr(), x.shape[0], out.data_ptr()))
    return out[:-1], float(out[-1].item())


def train(ab: Absorber, x, t, *, epochs: int = 4, batch: int = 8192, lr: float = 2e-3,
          seed: int = 0, params0=None, log=None) -> np.ndarray:
    """Adam on mini-batches drawn without replacement each epoch (seeded);
    gradients and updates by the device kernels.  Returns FP32 parameters."""
    import torch
    dev = x.device
    p = torch.from_numpy(init_params(seed) if params0 is None else np.asarray(params0, np.float32)).to(dev)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    g = torch.empty(num_params() + 1, dtype=torch.float64, device=dev)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    n = x.shape[0]
    step = 0
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen).to(dev)
        lr_ep = lr * (0.5 ** ep)
        losses = []
        for s0 in range(0, n - batch + 1 if n >= batch else 1, batch):
            idx = perm[s0:s0 + batch]
            xb = x.index_select(0, idx).contiguous()
            tb = t.index_select(0, idx).contiguous()
            _check(ab, ab.lib.b200fe_mlp_grad(ab.handle, p.data_ptr(), xb.data_ptr(), tb.data_ptr(),
                                              xb.shape[0], g.data_ptr()))
            step += 1
            _check(ab, ab.lib.b200fe_mlp_adam(ab.handle, p.data_ptr(), m.data_ptr(), v.data_ptr(),
                                              g.data_ptr(), step, lr_ep))
            if step % 50 == 0:
                losses.append(float(g[-1].item()))
        if log is not None:
            log(f"epoch {ep}: steps {step} mean loss {np.mean(losses) if losses else float('nan'):.5f}")
    return p.cpu().numpy()


def collect_samples(ab: Absorber, v, group_ids, num_groups, weights=None, *, tol: float = 1e-11,
                    capacity: int | None = None):
    """Features (count, 8) and targets (count, 4) of every level of the
    non-primary dims and every column, from the plain FP64 solver on this
    problem (device tensors as Absorber.absorb_device).  Returns
    (features, targets, result)."""
    import torch
    cols, n = v.shape
    G = np.ascontiguousarray(num_groups, dtype=np.int32)
    cap = capacity if capacity is not None else int(G.sum()) * cols
    feat = torch.empty((cap, N_FEATURES), dtype=torch.float32, device=v.device)
    targ = torch.empty((cap, 4), dtype=torch.float32, device=v.device)
    out = torch.empty_like(v)
    o = make_options(tol=tol, precision="fp64", tolerance_mode="strict-residual")
    r = _lib.Result()
    cnt = ctypes.c_int64(0)
    rc = ab.lib.b200fe_warmstart_samples(
        ab.handle, v.data_ptr(), n, cols, len(group_ids),
        _ptr_array([g.data_ptr() for g in group_ids]), G.ctypes.data,
        None if weights is None else weights.data_ptr(), ctypes.byref(o), out.data_ptr(),
        feat.data_ptr(), targ.data_ptr(), cap, ctypes.byref(cnt), ctypes.byref(r))
    if rc not in (_lib.OK, _lib.NOT_CONVERGED):
        raise ab._err(rc)
    k = int(cnt.value)
    return feat[:k], targ[:k], r


def set_warm_start(ab: Absorber, params, mode: int = MODE_START):
    """Install trained parameters in the absorber's context (mode bits:
    1 start from the prediction, 2 scale the Jacobi diagonal); None turns it off."""
    if params is None:
        _check(ab, ab.lib.b200fe_warmstart_set(ab.handle, None, 0))
        return
    p = np.ascontiguousarray(params, dtype=np.float32)
    if p.size != num_params():
        raise ValueError(f"expected {num_params()} parameters, got {p.size}")
    _check(ab, ab.lib.b200fe_warmstart_set(ab.handle, p.ctypes.data, int(mode)))


def load_trained(path=None) -> np.ndarray | None:
    """The parameters trained by train_warmstart.py (None when absent)."""
    f = Path(path) if path is not None else TRAINED
    if not f.exists():
        return None
    with np.load(f) as z:
        return np.asarray(z["params"], dtype=np.float32)
