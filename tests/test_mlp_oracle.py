"""The FP64 checker of the warm-start network against central finite differences (CPU)."""
from __future__ import annotations

import numpy as np

from oracle import mlp_oracle


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = [5, 7, 6, 1]
    count = sum(dims[l + 1] * dims[l] + dims[l + 1] for l in range(len(dims) - 1))
    p = rng.normal(scale=0.5, size=count)
    x = rng.normal(size=(23, dims[0]))
    t = rng.normal(size=23)
    loss, g = mlp_oracle.loss_and_gradients(p, dims, x, t)
    h = 1e-6
    num = np.empty_like(p)
    for k in range(count):
        e = np.zeros(count)
        e[k] = h
        num[k] = (mlp_oracle.loss_and_gradients(p + e, dims, x, t)[0] -
                  mlp_oracle.loss_and_gradients(p - e, dims, x, t)[0]) / (2 * h)
    assert np.max(np.abs(num - g)) <= 1e-7 * max(1.0, np.max(np.abs(g)))
    assert loss == float(np.mean((mlp_oracle.forward(p, dims, x)[-1][:, 0] - t) ** 2))
