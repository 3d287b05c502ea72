"""KPM moments on the GPU against the oracle (same seeded Rademacher vectors)."""
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import sma_oracle as O  # noqa: E402
from sparse_matrix_algorithms_b200 import matrices as M  # noqa: E402

pytestmark = pytest.mark.gpu


def test_kpm_moments_match_oracle(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(10, 16.5, 0)
    smin, smax = O.gershgorin_bounds(A)
    mu, pv = S.kpm_moments(A, 64, 8, smin=smin, smax=smax, seed=4, per_vector=True)
    mo, pvo = O.kpm_moments(A, 64, 8, 4, smin, smax, per_vector=True)
    assert mu[0] == 1.0
    np.testing.assert_allclose(pv, pvo, rtol=0, atol=1e-11)
    np.testing.assert_allclose(mu, pv.mean(axis=1), rtol=0, atol=1e-15)
    for a, b in [(-1.0, 1.0), (2.0, 6.0)]:
        assert abs(S.kpm_count(mu, A.shape[0], smin, smax, a, b) -
                   O.kpm_count(mu, A.shape[0], smin, smax, a, b)) <= 1e-9 * A.shape[0]


@pytest.mark.parametrize("M_", [1, 2, 7, 8])
def test_kpm_moments_diagonal_exact(lib_built, M_):
    import sparse_matrix_algorithms_b200 as S

    lam = np.linspace(-2.0, 3.0, 513)
    A = sp.diags(lam).tocsr()
    mu = S.kpm_moments(A, M_, 5, smin=-2.5, smax=3.5, seed=1)
    x = (lam - 0.5) / 3.0
    exact = np.array([np.mean(np.cos(k * np.arccos(x))) for k in range(M_)])
    np.testing.assert_allclose(mu, exact, rtol=0, atol=1e-12)


def test_kpm_stencil_equals_csr(lib_built):
    """The Anderson stencil's products are bit-identical to the CSR matrix's."""
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(16, 16.5, 2)
    smin, smax = O.gershgorin_bounds(A)
    m1 = S.kpm_moments(A, 128, 4, smin=smin, smax=smax)
    m2 = S.kpm_moments(S.AndersonOperator(16, 16.5, 2), 128, 4, smin=smin, smax=smax)
    np.testing.assert_array_equal(m1, m2)


def test_kpm_count_tracks_dense_count(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(12, 16.5, 0)
    lam = np.linalg.eigvalsh(A.toarray())
    smin, smax = O.gershgorin_bounds(A)
    mu = S.kpm_moments(A, 512, 64, smin=smin, smax=smax)
    for a, b in [(-0.5, 0.5), (-4.0, -2.0)]:
        exact = int(np.sum((lam >= a) & (lam <= b)))
        est = S.kpm_count(mu, A.shape[0], smin, smax, a, b)
        assert abs(est - exact) <= 0.1 * exact + 4, (a, b, est, exact)
