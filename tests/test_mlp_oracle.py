"""CPU: the FP64 model oracle against central finite differences."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    F, B = 7, 9
    P = M.H * F + M.H + M.H * M.H + M.H + M.H + 1
    p = rng.normal(0, 0.3, P)
    X = rng.normal(0, 1, (B, F))
    y = rng.normal(0, 1, B)
    _, g = M.loss_grad(p, X, y)
    idx = rng.choice(P, size=60, replace=False)
    idx[-1] = P - 1  # the output bias
    eps = 1e-6
    for i in idx:
        e = np.zeros(P)
        e[i] = eps
        num = (M.loss_grad(p + e, X, y)[0] - M.loss_grad(p - e, X, y)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 * max(1.0, abs(num)), (i, num, g[i])
