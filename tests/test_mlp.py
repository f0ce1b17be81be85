"""CPU checks of the warm-start network's oracle (oracle/mlp_oracle.py).

The backward formulas are checked against central finite differences of the
exact FP64 network (no BF16 rounding); the BF16 rounding helper against known
values; Adam against its textbook first step.  The device kernels are checked
against this oracle in tests/test_gpu_learned.py.
"""

import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding_known_values():
    vals = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -2.5, 0.0, 3.0e38])
    r = mo.bf16(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # halfway: ties to even
    assert r[2] == 1.0 + 2.0 ** -7          # above halfway: rounds up
    assert r[3] == -2.5 and r[4] == 0.0
    assert np.isfinite(r[5])


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = mo.init_params(1).astype(np.float64)
    p += 0.05 * rng.standard_normal(p.size)  # nonzero output layer and biases
    X = rng.standard_normal((40, mo.N_IN))
    T = np.column_stack([rng.standard_normal((40, 2)), rng.uniform(0.5, 1.5, (40, 2))])
    _, g = mo.loss_and_grad(p, X, T, rounding=False)
    idx = rng.choice(p.size, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        lp, _ = mo.loss_and_grad(p + e, X, T, rounding=False)
        lm, _ = mo.loss_and_grad(p - e, X, T, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_adam_first_step_moves_by_lr():
    p = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, 0.0])
    p1, m, v = mo.adam_step(p, g, np.zeros(4), np.zeros(4), 1, 0.01)
    assert np.allclose(p1[:3], -0.01 * np.sign(g[:3]), rtol=1e-6)
    assert p1[3] == 0.0


def test_parameter_layout():
    assert mo.N_PARAMS == 64 * 8 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 2 * 64 + 2
    P = mo.unpack(np.arange(mo.N_PARAMS, dtype=np.float64))
    assert P["W1"][0, 1] == 1 and P["b4"][-1] == mo.N_PARAMS - 1
