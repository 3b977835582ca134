"""The learned closure's numpy oracle (oracle/mlp.py) pinned by central finite
differences of its own loss; the GPU kernels are then checked against it."""
import numpy as np

from oracle import mlp


def _params(seed=0):
    rng = np.random.default_rng(seed)
    n = mlp.N_HID * mlp.N_IN + mlp.N_HID + mlp.N_HID * mlp.N_HID + mlp.N_HID + mlp.N_HID + 1
    return rng.normal(0.0, 0.3, n)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _params()
    X = rng.normal(0.0, 1.0, (64, mlp.N_IN))
    Y = rng.uniform(0.0, 3.0, 64)
    _, g = mlp.loss_and_grad(p, X, Y)
    h = 1e-6
    idx = rng.choice(p.size, 60, replace=False)
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp.loss_and_grad(pp, X, Y)[0] - mlp.loss_and_grad(pm, X, Y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_oracle_forward_is_positive_and_smooth():
    p = _params(2)
    X = np.random.default_rng(3).normal(0.0, 1.0, (100, mlp.N_IN))
    y, _ = mlp.forward(p, X)
    assert np.all(y > 0.0) and np.all(np.isfinite(y))
