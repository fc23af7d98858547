"""The numpy perceptron oracle's gradient against central finite
differences (no GPU)."""
import numpy as np

import mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    dims = [2, 7, 5, 3]
    n = sum(a * b + b for a, b in zip(dims[:-1], dims[1:]))
    p = rng.normal(0, 0.3, n)
    x = rng.uniform(-1, 1, (11, 2))
    t = rng.normal(0, 1, (11, 3))
    _, g = mo.loss_and_grad(p, dims, 3.0, x, t)
    h = 1e-6
    fd = np.zeros(n)
    for i in range(n):
        e = np.zeros(n)
        e[i] = h
        fd[i] = (mo.loss_and_grad(p + e, dims, 3.0, x, t)[0] -
                 mo.loss_and_grad(p - e, dims, 3.0, x, t)[0]) / (2 * h)
    assert np.max(np.abs(fd - g)) <= 1e-7 * max(1.0, np.max(np.abs(g)))
