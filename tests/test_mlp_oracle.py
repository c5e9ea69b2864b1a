"""The NumPy restatement of the early-termination network (its gradient oracle) is itself right."""

from __future__ import annotations

import numpy as np

from oracle import mlp


def test_gradients_match_finite_differences() -> None:
    rng = np.random.default_rng(0)
    p = mlp.init_params(1).astype(np.float64)
    X = rng.standard_normal((64, mlp.F))
    y = rng.standard_normal(64)
    g = mlp.gradients(p, X, y, round_weights=False, dtype=np.float64)
    eps = 1e-6
    for idx in rng.choice(mlp.NPARAM, 60, replace=False):
        a, b = p.copy(), p.copy()
        a[idx] += eps
        b[idx] -= eps
        fd = (mlp.loss(a, X, y, round_weights=False, dtype=np.float64)
              - mlp.loss(b, X, y, round_weights=False, dtype=np.float64)) / (2 * eps)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(fd), (idx, fd, g[idx])


def test_bf16_rounding_is_nearest_even() -> None:
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 2**-7, 1.0 + 3 * 2**-8, -2.5, 3.0e38], np.float32)
    r = mlp.bf16_round(x)
    np.testing.assert_array_equal(r[:4], [1.0, 1.0, 1.0 + 2**-7, 1.0 + 2**-6])
    assert r[4] == -2.5


def test_adam_step_moves_against_the_gradient() -> None:
    p = np.zeros(4)
    g = np.array([1.0, -1.0, 0.0, 2.0])
    q, m, v = mlp.adam_step(p, np.zeros(4), np.zeros(4), g, 1, 0.1)
    np.testing.assert_allclose(q, [-0.1, 0.1, 0.0, -0.1], atol=1e-6)
