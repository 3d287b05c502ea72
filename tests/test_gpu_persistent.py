"""The persistent (one cooperative launch) Clenshaw filter against the step-by-step one.

Both evaluate the same recurrence with the same FMA order, so filter outputs and whole
solves must agree bit for bit; `SMA_PERSISTENT=1` selects the persistent kernel for the
contexts created while it is set.
"""
import numpy as np
import pytest

from sparse_matrix_algorithms_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _contexts(S, monkeypatch):
    base = S.Context(0)
    monkeypatch.setenv("SMA_PERSISTENT", "1")
    pers = S.Context(0)
    monkeypatch.delenv("SMA_PERSISTENT")
    return base, pers


@pytest.mark.parametrize("precision,b", [("fp64", 32), ("fp64", 13), ("fp32", 48), ("fp32", 7)])
def test_persistent_filter_bit_identical(lib_built, monkeypatch, precision, b):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(20, 16.5, 1)
    base, pers = _contexts(S, monkeypatch)
    ob, op = S.SparseOperator(A, base), S.SparseOperator(A, pers)
    smin, smax = ob.gershgorin_bounds()
    Q = M.splitmix_normal(3, A.shape[0], b)
    for K in (1, 40, 333):
        c = S.build_coeffs(K, smin, smax, 0.1, -0.3, 0.5, "step")
        Y0 = S.apply_poly_block(ob, Q, c, smin, smax, precision=precision)
        Y1 = S.apply_poly_block(op, Q, c, smin, smax, precision=precision)
        np.testing.assert_array_equal(Y0, Y1)


def test_persistent_polfed_and_chebyshev_bit_identical(lib_built, monkeypatch):
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(14, 5.0, 1)
    lam_all = np.linalg.eigvalsh(A.toarray())
    mid = int(np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1]))))
    emin = 0.5 * (lam_all[mid - 16] + lam_all[mid - 15])
    emax = 0.5 * (lam_all[mid + 14] + lam_all[mid + 15])
    base, pers = _contexts(S, monkeypatch)
    out = []
    for ctx in (base, pers):
        op = S.SparseOperator(A, ctx)
        smin, smax = op.gershgorin_bounds()
        st = {}
        lp, Xp, rp = S.polfed(op, 30, 900, s=16, smin=smin, smax=smax, sigma=0.5 * (emin + emax),
                              emin=emin, emax=emax, mmax=8, window_type="delta", stats=st)
        lc, Xc, rc = S.chebyshev_poly_real_symm_sparse(
            S.MatrixFreeRealSymOp(A.shape[0], None, op), emin, emax, smin=smin, smax=smax,
            m0=48, degree=1500, maxiter=6, precision="mixed")
        out.append((lp, Xp, rp, lc, Xc, rc, st["graph_replays"]))
    for a, b in zip(out[0][:6], out[1][:6]):
        np.testing.assert_array_equal(a, b)
    assert out[0][6] > 0 and out[1][6] == 0  # graphs on the step-by-step path only


def test_bounded_barrier_reports_timeout_and_context_survives(lib_built):
    """Failure detection without a fault: the grid barrier waits for a CTA that was never
    launched, gives up after its wait limit (10 ms of elapsed time), sets the error flag and returns; the
    host reads SMA_ERR_TIMEOUT and the context keeps working."""
    import ctypes

    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    ctx = S.Context(0)
    obs = ctypes.c_int64(-1)
    L.check(L.load().sma_selftest_barrier_timeout(ctx.handle, ctypes.byref(obs)))
    assert obs.value == L.SMA_ERR_TIMEOUT
    A = M.anderson3d(8, 16.5, 0)
    op = S.SparseOperator(A, ctx)
    smin, smax = op.gershgorin_bounds()
    Q = M.splitmix_normal(1, A.shape[0], 8)
    c = S.build_coeffs(50, smin, smax, 0.0, -0.5, 0.5, "step")
    Y = S.apply_poly_block(op, Q, c, smin, smax)
    assert np.isfinite(Y).all() and np.abs(Y).max() > 0
