"""GPU parity of the hot path: the block Clenshaw filter (apply_poly_block!) and the
sparse block product, through the C ABI, against the CPU oracle on identical inputs.

Tolerances: FP64 results agree with the oracle to 1e-12 relative to the block's
magnitude (the GPU fuses multiply-adds, the oracle rounds twice, and the recurrence
runs K steps).  The FP32 filter is compared with the FP64 oracle at 2e-4 relative.
"""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import sma_oracle as O
from sparse_matrix_algorithms_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _ragged(n, seed):
    """Symmetric matrix with empty, short and long rows (ragged CSR)."""
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for i in range(n):
        k = [0, 1, 2, 5, 13][i % 5]
        js = rng.integers(0, n, size=k)
        rows += [i] * k
        cols += list(js)
    A = sp.coo_matrix((rng.uniform(-1, 1, len(rows)), (rows, cols)), shape=(n, n)).tocsr()
    A = A + A.T
    A.setdiag(np.where(np.arange(n) % 7 == 3, 0.0, rng.uniform(-2, 2, n)))
    A.eliminate_zeros()
    return M._canonical(A)


MATRICES = {
    "lap1d": lambda: M.lap1d(700),
    "anderson_L8": lambda: M.anderson3d(8, 16.5, 2),
    "xxz_L12": lambda: M.xxz_sz0(12, 5.0, 1),
    "ragged": lambda: _ragged(333, 4),
}


def _bounds(A):
    return O.gershgorin_bounds(A)


@pytest.mark.parametrize("name", sorted(MATRICES))
@pytest.mark.parametrize("b", [1, 2, 3, 8, 17, 32, 64, 100])
def test_filter_fp64_matches_oracle(lib_built, name, b):
    import sparse_matrix_algorithms_b200 as S

    A = MATRICES[name]()
    smin, smax = _bounds(A)
    Q = M.splitmix_normal(b, A.shape[0], b)
    for K, window in [(0, "step"), (1, "delta"), (2, "step"), (37, "smooth"), (160, "step")]:
        c = O.build_coeffs(K, smin, smax, 0.1, -0.4, 0.3, window, True)
        ref = O.apply_poly_block(A, Q, c, smin, smax)
        got = S.apply_poly_block(A, Q, c, smin, smax)
        scale = max(np.abs(ref).max(), np.abs(Q).max())
        assert np.abs(got - ref).max() <= 1e-12 * scale, (K, window)


@pytest.mark.parametrize("name,b", [("anderson_L28", 8), ("anderson_L28", 32), ("xxz_L18", 32),
                                    ("xxz_L18", 48), ("xxz_L18", 6)])
def test_filter_all_autotuner_candidates_match_oracle(lib_built, name, b):
    """Operators with n >= 20000 are autotuned online: the first 2 x (candidates) steps of
    the recurrence each run a different kernel configuration (all three families), so
    the result checks every configuration on real work."""
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(28, 16.5, 9) if name == "anderson_L28" else M.xxz_sz0(18, 5.0, 1)
    smin, smax = _bounds(A)
    op = S.SparseOperator(A)
    Q = M.splitmix_normal(5, A.shape[0], b)
    c = O.build_coeffs(90, smin, smax, 0.0, -0.3, 0.3, "step", True)
    ref = O.apply_poly_block(A, Q, c, smin, smax)
    for _ in range(2):  # tuning run, then the chosen configuration
        got = S.apply_poly_block(op, Q, c, smin, smax)
        assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), np.abs(Q).max())
    got32 = S.apply_poly_block(op, Q, c, smin, smax, precision="fp32")
    got32 = S.apply_poly_block(op, Q, c, smin, smax, precision="fp32")
    assert np.abs(got32 - ref).max() <= 2e-4 * np.abs(ref).max()


@pytest.mark.parametrize("b", [1, 4, 6, 32, 96])
def test_filter_fp32_close_to_oracle(lib_built, b):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(8, 16.5, 2)
    smin, smax = _bounds(A)
    Q = M.splitmix_normal(7, A.shape[0], b)
    c = O.build_coeffs(120, smin, smax, 0.0, -0.5, 0.5, "step", True)
    ref = O.apply_poly_block(A, Q, c, smin, smax)
    got = S.apply_poly_block(A, Q, c, smin, smax, precision="fp32")
    assert np.abs(got - ref).max() <= 2e-4 * np.abs(ref).max()


def test_identity_filter_returns_q(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(10, 3.0, 5)
    Q = M.splitmix_normal(1, A.shape[0], 16)
    c = O.cheb_window_coeffs(-1.0, 1.0, 80, jackson=True)
    Y = S.apply_poly_block(A, Q, c, *_bounds(A))
    assert np.abs(Y - Q).max() < 1e-12 * np.abs(Q).max()


def test_lap1d_stencil_operator_matches_csr_oracle(lib_built):
    import sparse_matrix_algorithms_b200 as S

    n = 1234
    op = S.Lap1dOperator(n)
    Q = M.splitmix_normal(9, n, 24)
    for K in [0, 1, 5, 200]:
        c = O.build_coeffs(K, 0.0, 4.0, 2.0, 1.9, 2.2, "delta", True)
        ref = O.apply_poly_block(M.lap1d(n), Q, c, 0.0, 4.0)
        got = S.apply_poly_block(op, Q, c, 0.0, 4.0)
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("Lsz", [5, 9, 28])
def test_anderson_stencil_matches_csr_kernel_and_oracle(lib_built, Lsz):
    """Matrix-free Anderson stencil: same terms in the same order as the CSR kernel."""
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(Lsz, 16.5, 3)
    st = S.AndersonOperator(Lsz, 16.5, 3)
    csr = S.SparseOperator(A)
    smin, smax = _bounds(A)
    for b, K in [(1, 7), (8, 60), (32, 130)]:
        Q = M.splitmix_normal(b, A.shape[0], b)
        c = O.build_coeffs(K, smin, smax, 0.0, -0.4, 0.4, "step", True)
        y_st = S.apply_poly_block(st, Q, c, smin, smax)
        y_csr = S.apply_poly_block(csr, Q, c, smin, smax)
        scale = max(np.abs(y_csr).max(), 1.0)
        assert np.abs(y_st - y_csr).max() <= 1e-15 * scale
        ref = O.apply_poly_block(A, Q, c, smin, smax)
        assert np.abs(y_st - ref).max() <= 1e-12 * max(np.abs(ref).max(), np.abs(Q).max())


@pytest.mark.parametrize("Lc", [4, 10, 14, 18])
def test_xxz_stencil_matches_oracle(lib_built, Lc):
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(Lc, 5.0, 1)
    st = S.XXZOperator(Lc, 5.0, 1)
    assert st.n == A.shape[0]
    smin, smax = _bounds(A)
    for b, K in [(2, 9), (16, 80)]:
        Q = M.splitmix_normal(b + 1, A.shape[0], b)
        c = O.build_coeffs(K, smin, smax, 0.0, -0.4, 0.4, "delta", True)
        ref = O.apply_poly_block(A, Q, c, smin, smax)
        got = S.apply_poly_block(st, Q, c, smin, smax)
        assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), np.abs(Q).max())


def _device(arr):
    import torch

    return torch.as_tensor(np.ascontiguousarray(arr), device="cuda")


def test_device_entry_with_padded_leading_dimension(lib_built):
    """sma_apply_poly_block_dev on row-major device blocks with ld > b."""
    import torch
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    A = M.anderson3d(7, 16.5, 1)
    n, b, ldq, ldy = A.shape[0], 10, 13, 16
    smin, smax = _bounds(A)
    op = S.SparseOperator(A)
    Q = M.splitmix_normal(4, n, b)
    Qpad = np.zeros((n, ldq))
    Qpad[:, :b] = Q
    dQ = _device(Qpad)
    dY = torch.full((n, ldy), 7.0, dtype=torch.float64, device="cuda")
    c = np.ascontiguousarray(O.build_coeffs(45, smin, smax, 0.0, -1.0, 1.5, "step", True))
    torch.cuda.synchronize()
    L.check(L.load().sma_apply_poly_block_dev(op.handle, c.ctypes.data, len(c) - 1, smin, smax,
                                              dQ.data_ptr(), ldq, dY.data_ptr(), ldy, b, 0))
    Y = dY.cpu().numpy()
    ref = O.apply_poly_block(A, Q, c, smin, smax)
    assert np.abs(Y[:, :b] - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.all(Y[:, b:] == 7.0)  # padding untouched


def test_spmm_dev_matches_scipy(lib_built):
    import torch
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    A = _ragged(500, 9)
    op = S.SparseOperator(A)
    X = M.splitmix_normal(2, 500, 33)
    dX = _device(X)
    dY = torch.empty((500, 33), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    L.check(L.load().sma_spmm_dev(op.handle, dX.data_ptr(), 33, dY.data_ptr(), 33, 33))
    assert np.abs(dY.cpu().numpy() - A @ X).max() < 1e-13 * np.abs(A @ X).max()


def test_empty_block_and_empty_matrix(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.lap1d(50)
    Y = S.apply_poly_block(A, np.zeros((50, 0)), [1.0, 0.5], 0.0, 4.0)
    assert Y.shape == (50, 0)
    E = sp.csr_matrix((0, 0))
    Y = S.apply_poly_block(E, np.zeros((0, 3)), [1.0, 0.5], 0.0, 4.0)
    assert Y.shape == (0, 3)


def test_invalid_csr_is_rejected_before_upload(lib_built):
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    ctx = S.context()
    colptr = np.array([0, 2, 3], dtype=np.int64)
    rowval = np.array([1, 0, 5], dtype=np.int64)  # unsorted and out of range
    nzval = np.ones(3)
    h = ctypes.c_void_p()
    rc = L.load().sma_op_create_csc(ctx.handle, 2, 3, colptr.ctypes.data, rowval.ctypes.data,
                                    nzval.ctypes.data, 0, 0, ctypes.byref(h))
    assert rc == L.SMA_ERR_ARG
    with pytest.raises(S.ArgumentError):
        S.SparseOperator(sp.csr_matrix(np.array([[1.0, 2.0], [0.0, 1.0]])), check_symmetric=True)


@pytest.mark.parametrize("precision,b", [("fp64", 32), ("fp64", 64), ("fp32", 64), ("fp32", 128)])
def test_autotuned_filter_bit_identical_to_untuned(lib_built, monkeypatch, capfd, precision, b):
    """The autotuner's trial steps run every candidate family on real recurrence steps --
    DIRECT, STAGED, ASYNC and BULK (rows staged by bulk copies onto an mbarrier) -- so a tuned
    filter equals an untuned one bit for bit only if every family computes the same bits.
    The BULK family must have been among the candidates."""
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(30, 16.5, 9)  # n = 27000: autotuned
    smin, smax = _bounds(A)
    Q = M.splitmix_normal(3, A.shape[0], b)
    c = O.build_coeffs(120, smin, smax, 0.0, -0.3, 0.3, "step", True)
    monkeypatch.setenv("SMA_AUTOTUNE_VERBOSE", "1")
    tuned = S.apply_poly_block(S.SparseOperator(A, S.Context(0)), Q, c, smin, smax, precision=precision)
    err = capfd.readouterr().err
    assert "bulk/" in err, err
    monkeypatch.setenv("SMA_AUTOTUNE", "0")
    plain = S.apply_poly_block(S.SparseOperator(A, S.Context(0)), Q, c, smin, smax, precision=precision)
    np.testing.assert_array_equal(tuned, plain)
