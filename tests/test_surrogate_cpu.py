"""CPU checks of the surrogate's oracle (no GPU): its analytic gradients agree
with finite differences, and its BF16 rounding is round-to-nearest-even."""
import numpy as np
import torch

import mlp_oracle as mo


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    a = (rng.standard_normal(10000) * 10.0 ** rng.integers(-8, 8, 10000)).astype(np.float32)
    a[:4] = [1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.0 - 2 ** -8, 0.0]   # ties to even
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(mo.bf16_round(a), ref)


def test_parameter_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    n_in, n = 5, 23
    P = mo.layout(n_in)["P"]
    p = rng.standard_normal(P) * 0.2
    x = rng.standard_normal((n, n_in))
    t = rng.standard_normal(n)
    _, g = mo.loss_and_grad(p, x, t, n_in, bf16=False, dtype=np.float64)
    idx = rng.choice(P, 60, replace=False)
    idx[:6] = [0, mo.layout(n_in)["b1"], mo.layout(n_in)["W2"] + 7, mo.layout(n_in)["b2"], mo.layout(n_in)["w3"],
               mo.layout(n_in)["b3"]]
    h = 1e-6
    for k in idx:
        q1, q2 = p.copy(), p.copy()
        q1[k] += h
        q2[k] -= h
        fd = (mo.loss_and_grad(q1, x, t, n_in, False, np.float64)[0]
              - mo.loss_and_grad(q2, x, t, n_in, False, np.float64)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_input_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    n_in = 19
    p = rng.standard_normal(mo.layout(n_in)["P"]) * 0.1
    x = rng.standard_normal((4, n_in))
    _, gx = mo.input_grad(p, x, n_in, bf16=False, dtype=np.float64)
    h = 1e-6
    for d in range(n_in):
        e = np.zeros(n_in)
        e[d] = h
        fd = (mo.forward(p, x + e, n_in, False, np.float64)[0] - mo.forward(p, x - e, n_in, False, np.float64)[0]) / (2 * h)
        np.testing.assert_allclose(gx[:, d], fd, rtol=1e-6, atol=1e-9)


def test_adam_first_step_moves_by_lr():
    p = np.zeros(10, np.float32)
    g = np.linspace(-1, 1, 10).astype(np.float32)
    q, m, v = mo.adam_step(p, np.zeros(10, np.float32), np.zeros(10, np.float32), g, 1, 1e-3)
    # bias-corrected first step: -lr * sign(g) (up to eps)
    np.testing.assert_allclose(q, -1e-3 * np.sign(g), atol=1e-8)
