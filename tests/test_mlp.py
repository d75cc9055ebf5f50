"""The warm-start network: the FP64 oracle's gradient against finite
differences (CPU), then the GPU kernels against the oracle: the forward pass
to 1e-5 relative, the gradient to 1e-4 relative (FP32 arithmetic on the
device, FP64 in the oracle), bit-for-bit repeatability, and training that
lowers the loss."""
import numpy as np
import pytest

import oracle_ffi as of
from edge_rs_b200 import mlp_gradient, mlp_init, mlp_predict, mlp_train

N_FEAT, N_OUT = 12, 3


def problem(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, N_FEAT)).astype(np.float32) * 2 + 1
    w = rng.standard_normal((N_FEAT, N_OUT)) * 0.3
    t = (np.tanh(x @ w) + 0.1 * np.sin(3 * x[:, :N_OUT])).astype(np.float32)
    params = mlp_init(seed + 1)
    mean, sd = x.mean(axis=0), x.std(axis=0)
    params[-24:-12] = mean
    params[-12:] = 1.0 / np.where(sd > 0, sd, 1.0)
    return params, x, t


def test_oracle_gradient_matches_finite_differences():
    params, x, t = problem(9)
    params = params.astype(np.float32)
    _, g = of.mlp_loss_grad(params, x, t)
    rng = np.random.default_rng(4)
    for p in rng.choice(5187, 40, replace=False):
        h = 1e-2 * max(abs(float(params[p])), 0.1)
        up, down = params.copy(), params.copy()
        up[p] += h
        down[p] -= h
        h_true = float(up[p]) - float(down[p])  # float32 spacing
        fd = (of.mlp_loss_grad(up, x, t)[0] - of.mlp_loss_grad(down, x, t)[0]) / h_true
        assert abs(fd - g[p]) <= 2e-3 * max(1.0, abs(g[p])) + 1e-6, (p, fd, g[p])


def test_oracle_gives_zero_gradient_to_the_normalisation():
    params, x, t = problem(5)
    _, g = of.mlp_loss_grad(params, x, t)
    assert np.all(g[-24:] == 0.0)


@pytest.mark.gpu
def test_gpu_forward_matches_the_oracle():
    params, x, _ = problem(1000)
    got = mlp_predict(params, x)
    want = of.mlp_predict(params, x)
    assert np.allclose(got, want, rtol=1e-5, atol=1e-5 * np.abs(want).max())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 63, 64, 65, 4000])
def test_gpu_gradient_matches_the_oracle(n):
    params, x, t = problem(n, seed=n)
    loss, g = mlp_gradient(params, x, t)
    loss_ref, g_ref = of.mlp_loss_grad(params, x, t)
    assert abs(loss - loss_ref) <= 1e-5 * max(1.0, abs(loss_ref))
    scale = np.abs(g_ref).max()
    assert np.allclose(g, g_ref, rtol=1e-4, atol=1e-5 * scale), np.abs(g - g_ref).max() / scale
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)


@pytest.mark.gpu
def test_gpu_gradient_and_training_repeat_bit_for_bit():
    params, x, t = problem(3000)
    a = mlp_gradient(params, x, t)[1]
    b = mlp_gradient(params, x, t)[1]
    assert np.array_equal(a, b)
    p1, l1 = mlp_train(x, t, params, epochs=5, batch=256, lr=1e-3, seed=3)
    p2, l2 = mlp_train(x, t, params, epochs=5, batch=256, lr=1e-3, seed=3)
    assert np.array_equal(p1, p2) and np.array_equal(l1, l2)


@pytest.mark.gpu
def test_gpu_training_lowers_the_loss():
    params, x, t = problem(8000, seed=2)
    before = of.mlp_loss_grad(params, x, t)[0]
    trained, losses = mlp_train(x, t, params, epochs=60, batch=512, lr=2e-3, seed=1)
    after = of.mlp_loss_grad(trained, x, t)[0]
    assert losses[-1] < losses[0]
    assert after < 0.25 * before, (before, after)
    # the normalisation is not trained
    assert np.array_equal(trained[-24:], params[-24:])
