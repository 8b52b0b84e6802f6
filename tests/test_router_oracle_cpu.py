"""The FP64 router oracle's backward pass is the true gradient (finite differences)."""
import numpy as np

from oracle.router_oracle import mlp_fp64


def test_router_oracle_gradients_by_finite_differences():
    d, h, c, n = 6, 8, 5, 10
    rng = np.random.default_rng(0)
    nparam = d * h + h + h * h + h + h * c + c
    W = rng.standard_normal(nparam) * 0.5
    x = rng.standard_normal((n, d))
    y = rng.integers(0, c, n)
    loss, g = mlp_fp64(W, x, y, d, h, c, rounding=False)
    flat = np.concatenate([a.ravel() for a in g])
    eps = 1e-6
    for i in range(nparam):
        Wp, Wm = W.copy(), W.copy()
        Wp[i] += eps
        Wm[i] -= eps
        fd = (mlp_fp64(Wp, x, y, d, h, c, rounding=False)[0] - mlp_fp64(Wm, x, y, d, h, c, rounding=False)[0]) / (2 * eps)
        assert abs(flat[i] - fd) < 1e-7, (i, flat[i], fd)
