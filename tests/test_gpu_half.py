"""Symmetric half storage (sma_op_create_csc_upper) against full storage.

Only the upper triangle is stored; the transposed half is added by atomic scatters, so
products agree with the full-storage kernel to rounding (not bit for bit), and solves must
return the dense spectrum's eigenvalues exactly as the full-storage solves do.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from sparse_matrix_algorithms_b200 import matrices as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["anderson", "xxz"])
def test_half_storage_products_and_filters(lib_built, which):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(12, 16.5, 3) if which == "anderson" else M.xxz_sz0(12, 4.0, 2)
    full, half = S.SparseOperator(A), S.SparseOperator(A, storage="upper")
    ndiag = int(np.count_nonzero(A.diagonal()))
    assert half.nnz_stored == (A.nnz - ndiag) // 2 + ndiag
    assert half.gershgorin_bounds() == pytest.approx(full.gershgorin_bounds(), rel=1e-14)
    smin, smax = full.gershgorin_bounds()
    Q = M.splitmix_normal(4, A.shape[0], 24)
    c = S.build_coeffs(300, smin, smax, 0.2, -0.5, 0.5, "step")
    Y0 = S.apply_poly_block(full, Q, c, smin, smax)
    Y1 = S.apply_poly_block(half, Q, c, smin, smax)
    assert np.abs(Y1 - Y0).max() <= 1e-12 * np.abs(Y0).max()
    Y0f = S.apply_poly_block(full, Q, c, smin, smax, precision="fp32")
    Y1f = S.apply_poly_block(half, Q, c, smin, smax, precision="fp32")
    assert np.abs(Y1f - Y0f).max() <= 1e-4 * np.abs(Y0f).max()


def test_half_storage_solvers_match_dense(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(9, 16.5, 6)
    lam_all = np.linalg.eigvalsh(A.toarray())
    nrm = max(abs(lam_all[0]), abs(lam_all[-1]))
    i0 = np.searchsorted(lam_all, 0.0) - 10
    emin = 0.5 * (lam_all[i0 - 1] + lam_all[i0])
    emax = 0.5 * (lam_all[i0 + 19] + lam_all[i0 + 20])
    half = S.SparseOperator(A, storage="upper", check_symmetric=True)
    smin, smax = half.gershgorin_bounds()
    lam, X, res = S.polfed(half, 20, 600, s=8, smin=smin, smax=smax, emin=emin, emax=emax,
                           window_type="step", mmax=12)
    assert lam.size == 20
    assert np.abs(lam - lam_all[i0:i0 + 20]).max() <= 1e-12 * nrm
    assert res.max() <= 1e-10 * nrm
    lc, Xc, rc = S.chebyshev_poly_real_symm_sparse(half, emin, emax, m0=40, degree=800, maxiter=8)
    assert lc.size == 20 and np.abs(lc - lam_all[i0:i0 + 20]).max() <= 1e-12 * nrm
    R = A @ Xc - Xc * lc  # eigenvectors of the full matrix
    assert np.linalg.norm(R, axis=0).max() <= 1e-10 * nrm


def test_half_storage_errors(lib_built):
    import sparse_matrix_algorithms_b200 as S

    B = sp.csr_matrix(np.array([[2.0, 1.0, 0.0], [0.5, 3.0, 0.0], [0.0, 0.0, 1.0]]))
    with pytest.raises(S.SMAError):
        S.SparseOperator(B, storage="upper", check_symmetric=True)
    A = M.anderson3d(6, 16.5, 0)
    with pytest.raises(S.ArgumentError):
        S.slice_spectrum(S.SparseOperator(A, storage="upper"), [(-0.1, 0.1)], [100], [16])
    with pytest.raises(S.ArgumentError):
        S.SparseOperator(A, storage="lower")


def test_half_storage_applies_lower_triangle_and_its_bounds(lib_built):
    """Half storage keeps the entries a_ij with i >= j of the CSC arrays (row i, column j),
    so the operator applied is L + L^T - D (L = tril(A), D its diagonal) whatever the other
    triangle held.  With check_symmetric off and a non-symmetric input, its products are
    those of L + L^T - D and its Gershgorin bounds are L + L^T - D's, which enclose that
    operator's spectrum."""
    import sparse_matrix_algorithms_b200 as S

    rng = np.random.default_rng(5)
    n = 700
    A = sp.random(n, n, density=0.01, random_state=5, format="csr") + sp.diags(rng.uniform(-2, 2, n))
    A = sp.csr_matrix(A)  # not symmetric
    L = sp.tril(A).tocsr()
    Aapp = (L + L.T - sp.diags(A.diagonal())).tocsr()
    half = S.SparseOperator(A, storage="upper")
    d = Aapp.diagonal()
    r = np.asarray(abs(Aapp).sum(axis=1)).ravel() - np.abs(d)
    lo, hi = half.gershgorin_bounds()
    assert lo == pytest.approx(float(np.min(d - r)), rel=1e-13, abs=1e-13)
    assert hi == pytest.approx(float(np.max(d + r)), rel=1e-13, abs=1e-13)
    ev = np.linalg.eigvalsh(Aapp.toarray())
    assert lo <= ev[0] and ev[-1] <= hi
    Q = M.splitmix_normal(2, n, 8)
    c = np.zeros(2)
    c[1] = 1.0  # p = T_1: Y = A_hat Q, which exposes the operator applied
    Y = S.apply_poly_block(half, Q, c, lo, hi)
    cen, dd = 0.5 * (lo + hi), 0.5 * (hi - lo)
    ref = (Aapp @ Q - cen * Q) / dd
    assert np.abs(Y - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
