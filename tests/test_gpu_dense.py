"""This library's FP64 tensor-core (DMMA) products, through the C ABI, against numpy in FP64:
the Gram X^T Y (split-n reduction) and the block update Y = alpha X B + beta Y, at the
shapes of the solvers -- tall skinny, ragged sizes (not multiples of the 64 x 64 / 128 x 64
tiles), odd leading dimensions and offsets (the 8-byte copy path) -- plus the in-place
X <- X B of CholQR.  Tolerance: 1e-13 relative to the product's scale (sum |x||y| over n).
The Gram is deterministic: two runs give the same bits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _gram(ctx, X, Y, m, k, C0=None, alpha=1.0, beta=0.0, ldc=None):
    import torch
    from sparse_matrix_algorithms_b200 import _lib as L

    n = X.shape[0]
    ldc = ldc or m
    Cd = _dev(np.zeros((k, ldc)) if C0 is None else C0)
    Xd, Yd = _dev(X), _dev(Y)
    torch.cuda.synchronize()
    L.check(L.load().sma_dense_gram_dev(ctx.handle, n, m, k, Xd.data_ptr(), X.shape[1],
                                        Yd.data_ptr(), Y.shape[1], Cd.data_ptr(), ldc, alpha, beta))
    return Cd.cpu().numpy()  # row j of this (k x ldc) array is column j of C


@pytest.mark.parametrize("n,m,k", [(262144, 64, 64), (50000, 200, 64), (9999, 37, 5),
                                   (3001, 130, 130), (100, 64, 64), (0, 8, 8)])
def test_gram_matches_numpy(lib_built, n, m, k):
    import sparse_matrix_algorithms_b200 as S

    ctx = S.context()
    rng = np.random.default_rng(n + m + k)
    ldx, ldy = m + (3 if m % 2 else 0), k
    X = rng.standard_normal((n, ldx))
    Y = rng.standard_normal((n, ldy))
    C = _gram(ctx, X, Y, m, k)
    ref = X[:, :m].T @ Y[:, :k]
    scale = (np.abs(X[:, :m]).T @ np.abs(Y[:, :k])).max() if n else 1.0
    assert np.abs(C[:, :m].T - ref).max() <= 1e-13 * max(scale, 1.0)
    assert np.array_equal(C, _gram(ctx, X, Y, m, k))  # deterministic


def test_gram_alpha_beta(lib_built):
    import sparse_matrix_algorithms_b200 as S

    ctx = S.context()
    rng = np.random.default_rng(1)
    n, m, k = 7000, 70, 40
    X, Y = rng.standard_normal((n, m)), rng.standard_normal((n, k))
    C0 = rng.standard_normal((k, m))
    C = _gram(ctx, X, Y, m, k, C0=C0, alpha=-0.5, beta=2.0)
    ref = -0.5 * (X.T @ Y) + 2.0 * C0.T
    assert np.abs(C.T - ref).max() <= 1e-12 * np.abs(ref).max()


def _update(ctx, X, Cm, p, transC, Y0, alpha, beta, m):
    import torch
    from sparse_matrix_algorithms_b200 import _lib as L

    n = X.shape[0]
    Xd, Cd, Yd = _dev(X), _dev(Cm), _dev(Y0)
    torch.cuda.synchronize()
    L.check(L.load().sma_dense_update_dev(ctx.handle, n, m, p, Xd.data_ptr(), X.shape[1],
                                          Cd.data_ptr(), max(Cm.shape[1], 1), int(transC),
                                          Yd.data_ptr(),
                                          Y0.shape[1], alpha, beta))
    return Yd.cpu().numpy()


@pytest.mark.parametrize("n,m,p", [(262144, 512, 64), (40000, 64, 64), (12345, 33, 70),
                                   (5000, 0, 16), (777, 1000, 200)])
@pytest.mark.parametrize("transC", [False, True])
def test_update_matches_numpy(lib_built, n, m, p, transC):
    import sparse_matrix_algorithms_b200 as S

    ctx = S.context()
    rng = np.random.default_rng(n + m + p + transC)
    X = rng.standard_normal((n, m + 1))  # ld = m + 1 (odd for even m: the 8-byte path)
    B = rng.standard_normal((m, p))
    if transC:  # C is p x m column-major: row i of the array = column i of C = row i of B
        Cm = np.ascontiguousarray(B)
    else:       # C is m x p column-major: row j of the array = column j of C
        Cm = np.ascontiguousarray(B.T)
    Y0 = rng.standard_normal((n, p + 2))
    Y = _update(ctx, X, Cm, p, transC, Y0, -1.0, 1.0, m)
    ref = Y0[:, :p] - X[:, :m] @ B
    scale = (np.abs(X[:, :m]) @ np.abs(B)).max() if m else 1.0
    assert np.abs(Y[:, :p] - ref).max() <= 1e-13 * max(scale, 1.0)
    assert np.array_equal(Y[:, p:], Y0[:, p:])  # columns beyond p untouched


def test_update_in_place_triangular_inverse(lib_built):
    """X <- X R^-1 in place (k <= 64, beta = 0: Y aliases X), the product that replaces the
    triangular solve of CholQR, against numpy."""
    import torch
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    ctx = S.context()
    rng = np.random.default_rng(7)
    n, k = 100000, 48
    X = rng.standard_normal((n, k))
    R = np.triu(rng.standard_normal((k, k))) + 5 * np.eye(k)
    Rinv = np.linalg.inv(R)
    Xd = _dev(X)
    Cd = _dev(np.ascontiguousarray(Rinv.T))  # column-major k x k
    torch.cuda.synchronize()
    L.check(L.load().sma_dense_update_dev(ctx.handle, n, k, k, Xd.data_ptr(), k, Cd.data_ptr(), k,
                                          0, Xd.data_ptr(), k, 1.0, 0.0))
    got = Xd.cpu().numpy()
    ref = X @ Rinv
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
