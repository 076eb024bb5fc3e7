"""The CPU oracle of the smoothing-length seed network (oracle/mlp.py).

Its backpropagation (without the BF16 rounding) must match central finite
differences of its own loss in FP64; its BF16 rounding must match round to
nearest even.  The GPU kernels' gradients are then checked against this
oracle (tests/test_gpu_hseed.py)."""
from __future__ import annotations

import numpy as np

import mlp


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -2.5e-3, 3.0e5], np.float32)
    r = mlp.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa wins (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[3] == 1.0078125
    assert abs(r[4] + 2.5e-3) <= 2.5e-3 * 2 ** -8 and abs(r[5] - 3.0e5) <= 3.0e5 * 2 ** -8


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(0)
    n = 300
    X = rng.normal(size=(n, 8)).astype(np.float32)
    y = rng.normal(size=n).astype(np.float32) * 0.01
    norm = np.concatenate([X.mean(0), 1.0 / X.std(0), [y.mean(), y.std()]]).astype(np.float32)
    p = rng.normal(size=mlp.N_PARAMS) * 0.3
    rows = mlp.sample_rows(128, 12345, n)
    loss, g = mlp.forward_backward(p, X, y, norm, rows, rounding=False)
    assert loss > 0
    eps = 1e-6
    idx = rng.choice(mlp.N_PARAMS, 60, replace=False)
    for k in idx:
        dp = np.zeros_like(p)
        dp[k] = eps
        lp, _ = mlp.forward_backward(p + dp, X, y, norm, rows, rounding=False)
        lm, _ = mlp.forward_backward(p - dp, X, y, norm, rows, rounding=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (k, fd, g[k])


def test_sample_rows_is_the_documented_hash():
    rows = mlp.sample_rows(5, 7, 1000, it=2)
    want = [((((2 * 5 + r) * 0x9E3779B97F4A7C15) % 2 ** 64) ^ 7) % 1000 for r in range(5)]
    assert rows.tolist() == want
