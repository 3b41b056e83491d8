"""The learned-order cost model on a GPU: forward pass and gradients of the
hand-written kernels against a numpy restatement, training, and the order
search with its score-order fallback."""
import numpy as np
import pytest

import cuts_b200 as cb
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _data(n, nin, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, nin)).astype(np.float32)
    w = rng.normal(size=nin)
    t = (np.tanh(X @ w) * 3 + 0.5 * X[:, 0] ** 2).astype(np.float32)
    return X, t


@pytest.mark.parametrize("nin", [1, 7, 16, 32])
def test_forward_matches_numpy(nin):
    m = cb.Mlp(nin, seed=nin)
    X, _ = _data(333, nin, 1)
    p = m.get_params()
    want, _ = mlp_ref.forward(p, X)
    got = m.predict(X)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("nin,n", [(16, 1), (16, 5), (16, 1000), (9, 257)])
def test_gradients_match_numpy(nin, n):
    """Every parameter's gradient (tolerance: float32 accumulation with atomics)."""
    m = cb.Mlp(nin, seed=3)
    X, t = _data(n, nin, 2)
    loss, g = m.loss_grad(X, t)
    wl, wg = mlp_ref.loss_grad(m.get_params(), X, t)
    np.testing.assert_allclose(loss, wl, rtol=1e-4)
    # float32 sums of n per-sample terms added by atomics in no fixed order:
    # absolute error grows with n and with the gradient's scale
    scale = np.abs(wg).max()
    np.testing.assert_allclose(g, wg, rtol=2e-3, atol=1e-4 * max(scale, 1.0) * max(1.0, n / 250))


def test_gradient_finite_difference():
    """Spot-check the numpy restatement itself against central differences."""
    nin = 5
    m = cb.Mlp(nin, seed=4)
    p = m.get_params().astype(np.float64)
    X, t = _data(40, nin, 5)
    _, g = mlp_ref.loss_grad(p, X, t)
    rng = np.random.default_rng(0)
    for i in rng.choice(p.size, 25, replace=False):
        e = np.zeros_like(p)
        e[i] = 1e-5
        fd = (mlp_ref.loss_grad(p + e, X, t)[0] - mlp_ref.loss_grad(p - e, X, t)[0]) / 2e-5
        assert abs(fd - g[i]) <= 1e-4 * max(1.0, abs(g[i]))


def test_training_reduces_loss():
    m = cb.Mlp(16, seed=0)
    X, t = _data(4000, 16, 6)
    l0, _ = m.loss_grad(X, t)
    l1 = m.train(X, t, epochs=300, batch=500, lr=3e-3)
    assert l1 < 0.2 * l0
    # set_params round trip
    p = m.get_params()
    m2 = cb.Mlp(16, seed=1)
    m2.set_params(p)
    np.testing.assert_allclose(m2.predict(X[:50]), m.predict(X[:50]), rtol=1e-6, atol=1e-6)
