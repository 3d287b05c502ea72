"""The planner-network oracle pinned on the CPU: analytic gradients against central
differences (FP64 network), BF16 round-to-nearest-even, and the plain window rule."""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import mlp_ref as R  # noqa: E402


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 3.0e-39],
                 dtype=np.float32)
    y = R.bf16_round(x)
    assert y[0] == 1.0
    assert y[1] == 1.0                      # tie -> even mantissa
    assert y[2] == 1.0 + 2.0 ** -6          # tie -> even mantissa
    assert y[3] == 1.0                      # below half an ulp
    assert y[4] == -2.5                     # exactly representable
    assert (y.view(np.uint32) & 0xFFFF).max() == 0


def test_oracle_gradient_against_finite_differences():
    rng = np.random.default_rng(0)
    i, h, o, B = 7, 16, 3, 9
    p = rng.normal(0, 0.4, R.sizes(i, h, o))
    X = rng.normal(0, 1, (B, i))
    T = rng.normal(0, 1, (B, o))
    w = rng.uniform(0.5, 1.5, (B, o))
    loss, g = R.loss_and_grad64(p, X, T, w, i, h, o)
    idx = rng.choice(p.size, 40, replace=False)
    fd = R.finite_difference_grad(p, X, T, w, i, h, o, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-7)
    assert loss > 0


def test_plain_rule_and_features():
    from sparse_matrix_algorithms_b200 import planner as P

    K, m0 = P.plain_rule(100.0, -10.0, 10.0, -0.5, 0.5)
    assert K == math.ceil(4 * math.pi * 10.0 / 1.0) and m0 == 168
    f = P.window_features(np.linspace(1, 0, 300), -10.0, 10.0, -5.0, 2.0)
    assert f.shape == (P.IN_DIM,) and f.dtype == np.float32
    assert f[P.N_MOMENTS] == -0.5 and abs(f[P.N_MOMENTS + 1] - 0.2) < 1e-7
    assert P.scaled(1000, 168, 0.5, 1.5, 10 ** 6) == (500, 256)
