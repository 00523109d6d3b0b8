"""The CPU MLP checker against finite differences (no GPU)."""
import numpy as np

import mlp_ref


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    widths = [5, 7, 6, 3]
    n = sum(widths[l] * widths[l + 1] + widths[l + 1] for l in range(3))
    p = rng.normal(0, 0.5, n)
    X = rng.normal(0, 1, (9, 5))
    T = rng.normal(0, 1, (9, 3))
    _, g = mlp_ref.loss_and_grad(p, widths, X, T, round=False)
    h = 1e-6
    fd = np.empty(n)
    for i in range(n):
        e = np.zeros(n)
        e[i] = h
        fd[i] = (mlp_ref.loss_and_grad(p + e, widths, X, T, False)[0]
                 - mlp_ref.loss_and_grad(p - e, widths, X, T, False)[0]) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-5, atol=1e-8)


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5], dtype=np.float32)
    np.testing.assert_array_equal(mlp_ref.bf16(a), [1.0, 1.0, 1.0 + 2 ** -6, 1.0, -2.5])
