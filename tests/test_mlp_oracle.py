"""The float64 MLP oracle of the learned models, pinned by finite differences (CPU)."""
import numpy as np
import pytest

from oracle import mlp


@pytest.mark.parametrize("out,loss_kind", [(1, 0), (24, 1)])
def test_oracle_gradient_matches_finite_differences(out, loss_kind):
    rng = np.random.default_rng(out)
    p = rng.normal(0, 0.3, mlp.n_params(out))
    x = rng.normal(0, 1, (16, mlp.FEAT))
    y = rng.random(16) if loss_kind == 0 else rng.integers(0, out, 16)
    w = rng.random(16) + 0.5
    loss, g = mlp.loss_and_grad(p, out, loss_kind, x, y, w)
    idx = rng.choice(p.size, 40, replace=False)
    eps = 1e-6
    for i in idx:
        q = p.copy(); q[i] += eps
        lp, _ = mlp.loss_and_grad(q, out, loss_kind, x, y, w)
        q[i] -= 2 * eps
        lm, _ = mlp.loss_and_grad(q, out, loss_kind, x, y, w)
        assert abs((lp - lm) / (2 * eps) - g[i]) < 1e-6 + 1e-4 * abs(g[i])
