"""The FP64 MLP oracle pinned by finite differences of its own loss (CPU only)."""
import numpy as np

from oracle import mlp_ref


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    n = sum(mlp_ref.DIMS[l + 1] * mlp_ref.DIMS[l] + mlp_ref.DIMS[l + 1] for l in range(4))
    p = rng.normal(0, 0.1, n)
    X = rng.normal(0, 1, (8, 16))
    Y = np.stack([rng.uniform(0, 1, 8), rng.uniform(0, .5, 8), rng.uniform(0, .5, 8), rng.normal(0, 1, 8)], axis=1)
    g = mlp_ref.gradients(p, X, Y, rounding=False)
    idx = rng.choice(n, 40, replace=False)
    h = 1e-6
    for i in idx:
        q = p.copy(); q[i] += h
        lp = mlp_ref.loss(q, X, Y, rounding=False)
        q[i] -= 2 * h
        lm = mlp_ref.loss(q, X, Y, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g).max()), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-9, -2.5, 3.14159265], dtype=np.float32)
    r = mlp_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2**-7 and r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-12
