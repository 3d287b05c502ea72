"""The KPM oracle pinned by known answers (CPU only).

* Diagonal matrix: z^T T_k(A_hat) z = sum_i T_k(lambda_hat_i) exactly for +-1 vectors, so
  the moments equal the normalized Chebyshev sums of the diagonal for any seed and R.
* Counts: the Jackson-damped density integral predicts the exact (dense) eigenvalue count
  of a window within its statistical and resolution error.
"""
import math
import os
import sys

import numpy as np
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import sma_oracle as O  # noqa: E402
from sparse_matrix_algorithms_b200 import matrices as M  # noqa: E402


def test_rademacher_block():
    Z = M.splitmix_rademacher(3, 1000, 4)
    assert Z.shape == (1000, 4)
    assert set(np.unique(Z)) == {-1.0, 1.0}
    assert abs(Z.mean()) < 0.1
    # column-major draw order: column j continues the stream of column j-1
    np.testing.assert_array_equal(M.splitmix_rademacher(3, 4000, 1)[:, 0], Z.T.reshape(-1))


def test_kpm_moments_diagonal_exact():
    lam = np.linspace(-3.0, 5.0, 301) ** 3 / 40.0
    A = sp.diags(lam)
    smin, smax = lam.min() - 0.1, lam.max() + 0.2
    mu = O.kpm_moments(A, 40, 3, 9, smin, smax)
    x = (lam - 0.5 * (smin + smax)) / (0.5 * (smax - smin))
    exact = np.array([np.mean(np.cos(k * np.arccos(x))) for k in range(40)])
    np.testing.assert_allclose(mu, exact, rtol=0, atol=1e-12)
    assert mu[0] == 1.0


def test_kpm_count_against_dense():
    A = M.anderson3d(10, 16.5, 0)
    lam = np.linalg.eigvalsh(A.toarray())
    smin, smax = O.gershgorin_bounds(A)
    mu = O.kpm_moments(A, 256, 32, 11, smin, smax)
    for a, b in [(-1.0, 1.0), (-3.0, -0.5), (2.0, 6.0)]:
        exact = int(np.sum((lam >= a) & (lam <= b)))
        est = O.kpm_count(mu, A.shape[0], smin, smax, a, b)
        assert abs(est - exact) <= 0.12 * exact + 4, (a, b, est, exact)
    # the whole interval holds everything
    assert abs(O.kpm_count(mu, A.shape[0], smin, smax, smin, smax) - A.shape[0]) < 1e-9 * A.shape[0]
