"""The per-column filter and the MIXED POLFED polish built on it.

* sma_apply_poly_block_percol_dev: every column runs its own polynomial; on a CSR matrix
  each column is bit-identical to sma_apply_poly_block_dev with that column's coefficients
  (FP64 and FP32), and within 1e-12 of the oracle's filter in FP64; model stencils agree
  with the oracle to 1e-12 as well.
* The identity behind the polish, p(A_hat) x = p(t) x + q_t(A_hat) (A - theta) x / d, with
  q_t applied in FP32: for a nearly converged vector the FP32 correction gives the filtered
  vector to FP64-level accuracy, while the FP32 filter applied to x itself does not.
"""
import numpy as np
import pytest

import sma_oracle as O
from sparse_matrix_algorithms_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _percol(op, C, smin, smax, Q, precision):
    import torch
    from sparse_matrix_algorithms_b200 import _lib as L

    dt = torch.float64 if precision == "fp64" else torch.float32
    Qd = torch.as_tensor(np.ascontiguousarray(Q), device="cuda").to(dt).contiguous()
    Yd = torch.empty_like(Qd)
    C = np.ascontiguousarray(C, dtype=np.float64)
    torch.cuda.synchronize()
    L.check(L.load().sma_apply_poly_block_percol_dev(op.handle, C.ctypes.data, C.shape[0] - 1,
                                                     smin, smax, Qd.data_ptr(), Yd.data_ptr(),
                                                     Q.shape[1], L.PRECISIONS[precision]))
    return Yd.double().cpu().numpy()


def _single(op, c, smin, smax, q, precision):
    import torch
    from sparse_matrix_algorithms_b200 import _lib as L

    dt = torch.float64 if precision == "fp64" else torch.float32
    Qd = torch.as_tensor(np.ascontiguousarray(q[:, None]), device="cuda").to(dt).contiguous()
    Yd = torch.empty_like(Qd)
    c = np.ascontiguousarray(c, dtype=np.float64)
    torch.cuda.synchronize()
    L.check(L.load().sma_apply_poly_block_dev(op.handle, c.ctypes.data, len(c) - 1, smin, smax,
                                              Qd.data_ptr(), 1, Yd.data_ptr(), 1, 1,
                                              L.PRECISIONS[precision]))
    return Yd.double().cpu().numpy()[:, 0]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_percol_filter_bit_identical_to_single_column_filters(lib_built, precision):
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(14, 5.0, 1)
    smin, smax = O.gershgorin_bounds(A)
    op = S.SparseOperator(A)
    b, K = 8, 150
    Q = M.splitmix_normal(5, A.shape[0], b)
    centres = np.linspace(-3.0, 3.0, b)
    C = np.stack([O.build_coeffs(K, smin, smax, s, s - 0.2, s + 0.2, "delta", True) for s in centres],
                 axis=1)
    Y = _percol(op, C, smin, smax, Q, precision)
    for j in range(b):
        yj = _single(op, C[:, j], smin, smax, Q[:, j], precision)
        assert np.array_equal(Y[:, j], yj), j
    if precision == "fp64":
        for j in (0, b - 1):
            yo = O.apply_poly_block(A, Q[:, j:j + 1], C[:, j], smin, smax)[:, 0]
            assert np.abs(Y[:, j] - yo).max() <= 1e-12 * max(1.0, np.abs(yo).max())


@pytest.mark.parametrize("stencil", ["anderson", "xxz"])
def test_percol_filter_stencils_match_oracle(lib_built, stencil):
    import sparse_matrix_algorithms_b200 as S

    if stencil == "anderson":
        A, op = M.anderson3d(10, 16.5, 4), S.AndersonOperator(10, 16.5, 4)
    else:
        A, op = M.xxz_sz0(12, 3.0, 2), S.XXZOperator(12, 3.0, 2)
    smin, smax = O.gershgorin_bounds(A)
    b, K = 8, 90
    Q = M.splitmix_normal(9, A.shape[0], b)
    C = np.stack([O.build_coeffs(K, smin, smax, s, s - 0.3, s + 0.3, "step", True)
                  for s in np.linspace(-2, 2, b)], axis=1)
    Y = _percol(op, C, smin, smax, Q, "fp64")
    for j in range(b):
        yo = O.apply_poly_block(A, Q[:, j:j + 1], C[:, j], smin, smax)[:, 0]
        assert np.abs(Y[:, j] - yo).max() <= 1e-12 * max(1.0, np.abs(yo).max())


def test_residual_form_in_fp32_reaches_fp64_accuracy(lib_built):
    """x = an eigenvector plus a 1e-6 perturbation.  p(A) x in FP32 directly carries
    FP32-level error; p(t) x + q_t(A_hat) r / d with q_t in FP32 matches the FP64 filter
    to ~1e-12."""
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(12, 5.0, 1)
    lam, V = np.linalg.eigh(A.toarray())
    smin, smax = O.gershgorin_bounds(A)
    c, d = 0.5 * (smin + smax), 0.5 * (smax - smin)
    i0 = int(np.argmin(np.abs(lam)))
    K = 400
    coeffs = O.build_coeffs(K, smin, smax, lam[i0], lam[i0] - 0.1, lam[i0] + 0.1, "step", False)
    rng = np.random.default_rng(3)
    b = 4
    X = V[:, i0:i0 + b] + 1e-6 * rng.standard_normal((A.shape[0], b))
    X /= np.linalg.norm(X, axis=0)
    theta = np.einsum("ij,ij->j", X, A @ X)
    R = A @ X - X * theta
    s = np.linalg.norm(R, axis=0)
    E, pt = zip(*[O.divided_difference(coeffs, (t - c) / d) for t in theta])
    E = np.stack(E, axis=1)
    op = S.SparseOperator(A)
    Z = _percol(op, E, smin, smax, R / s, "fp32")
    Y_res = X * np.array(pt) + Z * (s / d)
    Y_ref = O.apply_poly_block(A, X, coeffs, smin, smax)
    Y32 = S.apply_poly_block(A, X, coeffs, smin, smax, precision="fp32")
    err_res = np.abs(Y_res - Y_ref).max() / np.abs(Y_ref).max()
    err_32 = np.abs(Y32 - Y_ref).max() / np.abs(Y_ref).max()
    assert err_res <= 1e-11
    assert err_32 >= 1e3 * err_res  # the direct FP32 filter is far less accurate
