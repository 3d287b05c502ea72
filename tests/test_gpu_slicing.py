"""Batched spectrum slicing on the GPU (sma_slice_solve).

The batched filter gives every window exactly the filtered block a single-window filter
gives it, so each window of a slicing run must reproduce, bit for bit, the matrix-free
Chebyshev solve of that window alone with the same seed, degree and width.  Eigenvalues
and counts are checked against a dense FP64 spectrum.
"""
import math

import numpy as np
import pytest

from sparse_matrix_algorithms_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _windows(lam_all, start, counts):
    """Contiguous windows holding counts[w] eigenvalues each, ends at mid-gaps."""
    wins, i = [], start
    for c in counts:
        wins.append((0.5 * (lam_all[i - 1] + lam_all[i]), 0.5 * (lam_all[i + c - 1] + lam_all[i + c])))
        i += c
    return wins


def _plain_rule(wins, smin, smax, counts, kmax=3000):
    """Degree ~ 4 pi d / width, width m0 = 2 count + 8 (multiple of 8)."""
    d = 0.5 * (smax - smin)
    deg = [min(kmax, int(math.ceil(4 * math.pi * d / (b - a)))) for a, b in wins]
    m0 = [int(8 * math.ceil((2 * c + 8) / 8)) for c in counts]
    return deg, m0


def _single(S, op, n, win, deg, m0, w, seed, precision, maxiter):
    a, b = win
    smin, smax = op.gershgorin_bounds()
    return S.chebyshev_poly_real_symm_sparse(
        S.MatrixFreeRealSymOp(n, None, op), a, b, smin=smin, smax=smax, sigma=0.5 * (a + b),
        m0=m0, degree=deg, maxiter=maxiter, seed=seed + w, precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_slicing_bit_identical_to_single_windows(lib_built, precision):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(12, 16.5, 0)
    n = A.shape[0]
    lam_all = np.linalg.eigvalsh(A.toarray())
    op = S.SparseOperator(A)
    smin, smax = op.gershgorin_bounds()
    mid = int(np.searchsorted(lam_all, 0.0))
    counts = [10, 20, 14]
    wins = _windows(lam_all, mid - 20, counts)
    deg, m0 = _plain_rule(wins, smin, smax, counts)
    st = {}
    lam, X, res, win = S.slice_spectrum(op, wins, deg, m0, maxiter=6, seed=5,
                                        precision=precision, stats=st)
    assert st["graph_replays"] > 0
    for w in range(len(wins)):
        l1, X1, r1 = _single(S, op, n, wins[w], deg[w], m0[w], w, 5, precision, 6)
        sel = win == w
        np.testing.assert_array_equal(lam[sel], l1)
        np.testing.assert_array_equal(res[sel], r1)
        np.testing.assert_array_equal(X[:, sel], X1)


def test_slicing_eigenvalues_against_dense(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(12, 16.5, 0)
    lam_all = np.linalg.eigvalsh(A.toarray())
    nrm = max(abs(lam_all[0]), abs(lam_all[-1]))
    op = S.SparseOperator(A)
    smin, smax = op.gershgorin_bounds()
    mid = int(np.searchsorted(lam_all, 0.0))
    counts = [8, 16, 12, 24, 6]
    start = mid - 30
    wins = _windows(lam_all, start, counts)
    deg, m0 = _plain_rule(wins, smin, smax, counts)
    lam, X, res, win = S.slice_spectrum(op, wins, deg, m0, maxiter=10)
    i = start
    for w, c in enumerate(counts):
        got = lam[win == w]
        assert got.size == c, (w, got.size, c)
        assert np.abs(got - lam_all[i:i + c]).max() <= 1e-12 * nrm
        assert res[win == w].max() <= 1e-10 * nrm
        i += c
    R = A @ X - X * lam  # the returned vectors are eigenvectors of A
    assert np.linalg.norm(R, axis=0).max() <= 1e-10 * nrm


def test_slicing_graph_and_eager_agree(lib_built):
    """Graph replay and eager launches give identical results (n above the autotuner's
    threshold, so the eager call also tunes the kernel for every active width)."""
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(28, 16.5, 3)
    op = S.SparseOperator(A)
    wins = [(-0.30, -0.22), (-0.22, -0.18), (-0.18, -0.05)]
    deg, m0 = [400, 700, 250], [16, 24, 40]
    sg, se = {}, {}
    lg, Xg, rg, wg = S.slice_spectrum(op, wins, deg, m0, maxiter=3, two_hit=False, tol=0.0,
                                      graph=True, stats=sg)
    le, Xe, re, we = S.slice_spectrum(op, wins, deg, m0, maxiter=3, two_hit=False, tol=0.0,
                                      graph=False, stats=se)
    assert sg["graph_replays"] == 2 and se["graph_replays"] == 0
    np.testing.assert_array_equal(lg, le)
    np.testing.assert_array_equal(rg, re)
    np.testing.assert_array_equal(Xg, Xe)
    np.testing.assert_array_equal(wg, we)
    assert sg["spmm_steps"] == se["spmm_steps"] == 3 * 701
    # one launch per recurrence index for all windows: summed active widths
    assert se["spmm_columns"] == 3 * (24 * 701 + 16 * 401 + 40 * 251)


def test_slicing_errors(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(6, 16.5, 0)
    op = S.SparseOperator(A)
    smin, smax = op.gershgorin_bounds()
    with pytest.raises(S.SMAError):
        S.slice_spectrum(op, [(smax + 1.0, smax + 2.0)], [100], [16])
    with pytest.raises(S.ArgumentError):
        S.slice_spectrum(op, [(-0.1, 0.1)], [100, 200], [16])
    with pytest.raises(S.ArgumentError):
        S.slice_spectrum(op, [(0.1, -0.1)], [100], [16])
    with pytest.raises(S.ArgumentError):
        S.slice_spectrum(S.AndersonOperator(6, 16.5, 0), [(-0.1, 0.1)], [100], [16])
