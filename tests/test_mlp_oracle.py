"""The learned tuner's CPU oracle (oracle/mlp_oracle.py) against finite
differences, so that it can stand as the checker of the CUDA kernels."""
import numpy as np

from oracle import mlp_oracle as M


def _problem(seed, n=23):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, M.PARAMS)
    X = rng.normal(0, 1, (n, M.IN))
    T = rng.normal(0, 1, (n, M.OUT))
    T[rng.random(T.shape) < 0.2] = np.nan
    return p, X, T


def test_gradient_matches_finite_differences():
    p, X, T = _problem(1)
    _, g = M.loss_grad(p, X, T, 0.1)
    eps = 1e-6
    rng = np.random.default_rng(2)
    for i in rng.choice(M.PARAMS, 200, replace=False):
        q = p.copy()
        q[i] += eps
        lp, _ = M.loss_grad(q, X, T, 0.1)
        q[i] -= 2 * eps
        lm, _ = M.loss_grad(q, X, T, 0.1)
        assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-5 * max(1.0, abs(g[i]))


def test_nan_targets_carry_no_loss():
    p, X, T = _problem(3)
    T[:] = np.nan
    loss, g = M.loss_grad(p, X, T, 1.0)
    assert loss == 0 and not g.any()


def test_adam_reduces_loss():
    p, X, T = _problem(4, n=64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    l0, _ = M.loss_grad(p, X, T, 1 / 64)
    for k in range(1, 300):
        _, g = M.loss_grad(p, X, T, 1 / 64)
        p, m, v = M.adam(p, g, m, v, k, 1e-2)
    l1, _ = M.loss_grad(p, X, T, 1 / 64)
    assert l1 < 0.5 * l0
