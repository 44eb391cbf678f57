"""The CPU float64 MLP restatement (oracle/mlp.py) pinned by finite differences,
so it can serve as the checker of the GPU gradients."""
import numpy as np

from oracle import mlp


def test_gradient_matches_central_differences():
    rng = np.random.default_rng(4)
    p = rng.normal(scale=0.3, size=mlp.NUM_PARAMS)
    norm = np.concatenate([rng.normal(size=16), rng.uniform(0.5, 2, 16), rng.normal(size=3), rng.uniform(0.5, 2, 3)])
    x = rng.normal(size=(40, 16))
    y = rng.normal(size=(40, 3))
    _, loss, g = mlp.forward_backward(p, norm, x, y)
    idx = rng.choice(mlp.NUM_PARAMS, size=60, replace=False)
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp = mlp.forward_backward(q, norm, x, y)[1]
        q[i] -= 2 * h
        lm = mlp.forward_backward(q, norm, x, y)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])
    assert mlp.NUM_PARAMS == 5443 and loss > 0
