"""The learned-densification network's CPU oracle: analytic gradients against central
finite differences in float64 (the network has no reference counterpart; this pins the
oracle the tensor-core kernels are checked against)."""
import numpy as np

from oracle import mlp as M


def _data(seed, n=40):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, M.IN))
    y = rng.integers(0, M.OUT, n)
    w = rng.uniform(0.5, 2.0, n)
    return x, y, w


def test_mlp_oracle_gradient_matches_finite_differences():
    theta = M.init_params(3)
    theta[M.NUM_PARAMS - 3:] = [0.1, -0.2, 0.05]
    x, y, w = _data(4)
    g = M.backward(theta, x, y, w)
    rng = np.random.default_rng(5)
    idx = rng.choice(M.NUM_PARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (M.loss(tp, x, y, w) - M.loss(tm, x, y, w)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_mlp_oracle_bf16_rounding_points():
    """bf16 rounding is round-to-nearest-even, and the bf16 forward stays within bf16
    precision of the float64 one."""
    assert M.bf16(np.array([1.0 + 2 ** -8]))[0] == 1.0          # tie to even
    assert M.bf16(np.array([1.0 + 3 * 2 ** -8]))[0] == 1.0 + 2 ** -6
    theta = M.init_params(1)
    x, _, _ = _data(2)
    p64, _ = M.forward(theta, x)
    p16, _ = M.forward(theta, x, bf16_like=True)
    assert np.abs(p64 - p16).max() < 2e-2
    assert np.allclose(p16.sum(1), 1.0)
