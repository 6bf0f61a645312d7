"""The double-precision MLP oracle's analytic gradient agrees with finite
differences (CPU only)."""
import numpy as np

from oracle import mlp_ref


def test_mlp_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    F, O, n = 5, 2, 7
    P = F * 64 + 64 + 2 * (64 * 64 + 64) + 64 * O + O
    p = rng.normal(0, 0.2, P)
    x = rng.normal(0, 1, (n, F))
    t = rng.normal(0, 1, (n, O))
    _, g = mlp_ref.loss_and_grad(p, x, t, F, O)
    eps = 1e-6
    for i in rng.choice(P, 60, replace=False):
        d = np.zeros(P)
        d[i] = eps
        fd = (mlp_ref.loss_only(p + d, x, t, F, O) - mlp_ref.loss_only(p - d, x, t, F, O)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])
