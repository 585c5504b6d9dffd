"""The surrogate's CUDA kernels (through the C ABI) against the CPU oracle
(oracle/mlp_oracle.py): forward pass, parameter gradients, input gradients and
Adam steps; plus training on a smooth target."""
import numpy as np
import pytest

import mlp_oracle as mo
from nonstationary_mra_b200.fit import Surrogate

pytestmark = pytest.mark.gpu

N_IN = 19


def data(seed, n):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, N_IN)).astype(np.float32)
    t = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.2 * np.sum(x ** 2, axis=1) / N_IN).astype(np.float32)
    return x, t


def test_forward_matches_oracle():
    net = Surrogate(N_IN, seed=1)
    x, _ = data(0, 77)
    y = net.predict(x)
    y_ref, _ = mo.forward(net.params(), x, N_IN)
    np.testing.assert_allclose(y, y_ref, rtol=1e-4, atol=1e-5)
    net.close()


def test_tensor_core_forward_many_tiles():
    # values only: the 128 x 128 layer runs on tcgen05 (128-sample tiles, more
    # tiles than SMs, a partial last tile); with input gradients the same network
    # runs on the FP32 cores -- the two agree to FP32 rounding, and both match the
    # oracle
    net = Surrogate(N_IN, seed=11)
    x, _ = data(5, 40000)
    y_tc = net.predict(x)
    y_fp32, _ = net.predict(x, with_grad=True)
    y_ref, _ = mo.forward(net.params(), x, N_IN)
    np.testing.assert_allclose(y_tc, y_fp32, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(y_tc, y_ref, rtol=1e-4, atol=1e-5)
    # a second call reuses the same buffers and barrier phases
    np.testing.assert_array_equal(net.predict(x[:333]), y_tc[:333])
    net.close()


def test_parameter_gradient_matches_oracle():
    net = Surrogate(N_IN, seed=2)
    x, t = data(1, 203)     # not a multiple of the 16-sample tile
    net.set_data(x, t)
    g, loss = net.grad()
    loss_ref, g_ref = mo.loss_and_grad(net.params(), x, t, N_IN)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    L = mo.layout(N_IN)
    for a, b in [("W1", "b1"), ("b1", "W2"), ("W2", "b2"), ("b2", "w3"), ("w3", "b3")]:
        np.testing.assert_allclose(g[L[a]:L[b]], g_ref[L[a]:L[b]], rtol=2e-3, atol=1e-6 * np.abs(g_ref).max())
    net.close()


def test_input_gradient_matches_oracle():
    net = Surrogate(N_IN, seed=3)
    x, _ = data(2, 40)
    y, gx = net.predict(x, with_grad=True)
    y_ref, gx_ref = mo.input_grad(net.params(), x, N_IN)
    np.testing.assert_allclose(y, y_ref, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(gx, gx_ref, rtol=1e-3, atol=1e-5 * np.abs(gx_ref).max())
    net.close()


def test_adam_steps_match_oracle():
    net = Surrogate(N_IN, seed=4)
    x, t = data(3, 128)
    net.set_data(x, t)
    p = net.params()
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    lr, steps = 1e-3, 5
    for k in range(1, steps + 1):
        _, g = mo.loss_and_grad(p, x, t, N_IN)
        p, m, v = mo.adam_step(p, m, v, g, k, lr)
    net.train(steps, lr)
    q = net.params()
    diff = np.abs(q - p)
    # Adam normalises each gradient entry: entries whose gradient is near a
    # rounding-level tie can differ by up to lr per step, the rest agree closely
    assert np.mean(diff <= 1e-6) > 0.995, np.mean(diff <= 1e-6)
    assert diff.max() <= 2 * lr * steps
    net.close()


def test_training_fits_a_smooth_target():
    net = Surrogate(N_IN, seed=5)
    x, t = data(4, 400)
    net.set_data(x, t)
    _, l0 = net.grad()
    l1 = net.train(3000, 2e-3)
    assert l1 < 0.05 * l0, (l0, l1)
    # deterministic: the same seed and data give the same parameters
    net2 = Surrogate(N_IN, seed=5)
    net2.set_data(x, t)
    net2.train(3000, 2e-3)
    np.testing.assert_array_equal(net.params(), net2.params())
    net.close()
    net2.close()


def test_trained_network_ranks_unseen_parameters():
    """What the network adds over the exact method alone: trained on exact
    (theta, loglik) pairs, it orders parameter vectors it has not seen by their
    exact log-likelihood without evaluating them (Spearman correlation), so the
    fitting loop can spend exact evaluations on its best candidates only."""
    from nonstationary_mra_b200 import api, partition, synth
    from nonstationary_mra_b200.fit import NonstationaryObjective
    rng = np.random.default_rng(21)
    cfg = synth.Config("s", 2048, 4, 4, 16, 1, 8, "uniform", 0.3, 21)
    xy, _ = synth.locations(cfg, rng)
    theta = synth.true_theta(cfg, rng)
    md = synth.model_from_theta(theta, 1)
    st = partition.build_by_program(xy[0], xy[1], np.zeros(cfg.n), 4, 4, 16, np.e / 100, distance=2)
    ctx = api.Context(st, md)
    ctx.set_theta()
    st.obs_value = ctx.sample_prior(rng.standard_normal(st.n_interior * st.r), rng.standard_normal(st.n_obs))
    ctx.set_obs_values(st.obs_value)
    obj = NonstationaryObjective(ctx, 0.0, float(np.log(0.1)))
    t0 = synth.theta_vector(theta)
    pts = t0 + rng.uniform(-0.4, 0.4, size=(264, N_IN))
    ll = np.array([obj.loglik(p) for p in pts])
    tr, te = slice(0, 200), slice(200, 264)
    scale = 0.4
    x = ((pts - t0) / scale).astype(np.float32)
    mu, sd = ll[tr].mean(), ll[tr].std()
    net = Surrogate(N_IN, seed=7)
    net.set_data(x[tr], ((ll[tr] - mu) / sd).astype(np.float32))
    net.train(3000, 2e-3)
    pred = net.predict(x[te])
    rank = lambda a: np.argsort(np.argsort(a))
    rho = np.corrcoef(rank(pred), rank(ll[te]))[0, 1]
    print(f"Spearman rank correlation on unseen parameters: {rho:.3f}")
    assert rho > 0.5, rho
    # the network's top quarter is better, by exact loglik, than the rest
    top = np.argsort(-pred)[:16]
    assert ll[te][top].mean() > ll[te].mean()
    net.close()
    ctx.close()
