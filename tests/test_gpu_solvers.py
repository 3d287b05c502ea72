"""GPU parity of the two solvers, through the C ABI (Python mirror), against
exactly known spectra (1D Laplacian, dense FP64 eigensolves) and the CPU oracle.

Criteria (from the reference's own checks and the acceptance rule of this port):
eigenvalue count inside [emin, emax] exact, |dlambda| <= 1e-12 * ||A||, relative
residual ||Ax - lambda x|| / ||A|| <= 1e-10 for the FP64 solvers.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import sma_oracle as O
from sparse_matrix_algorithms_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _norm2(lam_all):
    return max(abs(lam_all[0]), abs(lam_all[-1]))


def _classify(lam_got, lam_ref, lam_all, tol=1e-8):
    """matched / legit extra / spurious (chebyshev_subspace_iteration.jl:918-979)."""
    got = np.sort(lam_got)
    matched = sum(np.min(np.abs(got - r)) <= tol for r in lam_ref) if got.size else 0
    legit = sum(np.min(np.abs(lam_all - g)) <= tol for g in got)
    return matched, legit, got.size - legit


def _window_with_gaps(lam_all, i_lo, i_hi):
    """[emin, emax] holding exactly lam_all[i_lo..i_hi], ends at mid-gaps."""
    return 0.5 * (lam_all[i_lo - 1] + lam_all[i_lo]), 0.5 * (lam_all[i_hi] + lam_all[i_hi + 1])


# ---------------------------------------------------------------------- Chebyshev
def test_chebyshev_sparse_lap1d_reference_harness(lib_built):
    """The reference's count test (chebyshev_subspace_iteration.jl:993-1023) on a small n."""
    import sparse_matrix_algorithms_b200 as S

    n, nev = 2000, 40
    emin, emax, sigma, lref, _ = M.lap1d_interval_by_count(n, nev)
    lam, X, res = S.chebyshev_poly_real_symm_sparse(
        M.lap1d(n), emin, emax, smin=0.0, smax=4.0, σ=sigma, m0=2 * nev, degree=128,
        maxiter=10, tol=1e-8, res_gate=1e-6, window_type="delta", two_hit=False)
    matched, legit, spurious = _classify(lam, lref, M.lap1d_exact_eigs(n))
    assert matched == nev and spurious == 0
    assert np.all(np.diff(lam) >= 0)
    assert res.max() < 1e-8
    # residuals recomputed on the host from the returned vectors
    A = M.lap1d(n)
    r = np.linalg.norm(A @ X - X * lam, axis=0)
    assert np.abs(r - res).max() < 1e-12


def test_chebyshev_matches_oracle_same_start_block(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(8, 16.5, 3)
    lam_all = np.linalg.eigvalsh(A.toarray())
    i_lo = np.searchsorted(lam_all, -0.6)
    emin, emax = _window_with_gaps(lam_all, i_lo, i_lo + 11)
    kw = dict(m0=24, degree=600, maxiter=6, window_type="step")
    lam_g, X_g, res_g = S.chebyshev_poly_real_symm_sparse(A, emin, emax, **kw)
    lam_o, X_o, res_o = O.chebyshev_poly_real_symm_sparse(A, emin, emax, **kw)
    assert lam_g.size == lam_o.size == 12
    nrm = _norm2(lam_all)
    assert np.abs(lam_g - lam_o).max() < 1e-12 * nrm
    assert np.abs(lam_g - lam_all[i_lo:i_lo + 12]).max() < 1e-12 * nrm
    assert res_g.max() < 1e-10 * nrm


def test_chebyshev_matrix_free_two_hit(lib_built):
    """Matrix-free overload (chebyshev_subspace_iteration.jl:771): device stencil operator,
    two_hit early exit."""
    import sparse_matrix_algorithms_b200 as S

    n, nev = 3000, 30
    emin, emax, sigma, lref, _ = M.lap1d_interval_by_count(n, nev)
    st = {}
    lam, X, res = S.chebyshev_poly_real_symm_sparse(
        None, n, emin, emax, matblock=S.Lap1dOperator(n), smin=0.0, smax=4.0, sigma=sigma,
        m0=60, degree=200, maxiter=20, tol=1e-10, window_type="delta", stats=st)
    matched, legit, spurious = _classify(lam, lref, M.lap1d_exact_eigs(n))
    assert matched == nev and spurious == 0
    assert 2 <= st["iterations"] < 20  # stopped early on two consecutive hits
    assert res.max() < 1e-9


def test_chebyshev_c1_anderson_L20_count_and_accuracy(lib_built):
    """Config C1: Anderson L=20 (n=8000), W=16.5, seed 0, window [-0.05, 0.05], m0=64,
    Gershgorin bounds, against the dense FP64 spectrum."""
    import sparse_matrix_algorithms_b200 as S
    from conftest import GOLDEN

    g = np.load(f"{GOLDEN}/anderson_L20_spectrum.npz")
    c = g["central"]
    count = int(((c >= -0.05) & (c <= 0.05)).sum())
    A = M.config_matrix("anderson_L20")
    lam, X, res = S.chebyshev_poly_real_symm_sparse(A, -0.05, 0.05, m0=64, degree=1500,
                                                    maxiter=8, window_type="delta", sigma=0.0)
    nrm = max(abs(float(g["lam_min"])), abs(float(g["lam_max"])))
    assert lam.size == count
    exact = c[(c >= -0.05) & (c <= 0.05)]
    assert np.abs(lam - exact).max() <= 1e-12 * nrm
    assert res.max() <= 1e-10 * nrm


# ---------------------------------------------------------------------- POLFED
def test_polfed_lap1d_stencil_reference_setup(lib_built):
    """polfed.jl:1243-1260 scaled down: lap1d_target_window, smin=0, smax=4, :delta."""
    import sparse_matrix_algorithms_b200 as S

    n, nev, s = 4000, 60, 16
    lam_all, i1, i2, emin, emax, sigma = M.lap1d_target_window(n, nev)
    Aop = S.MatrixFreeRealSymOp(n, None, S.Lap1dOperator(n))
    lam, X, res = S.polfed(Aop, nev, 300, s=s, smin=0.0, smax=4.0, sigma=sigma, emin=emin,
                           emax=emax, tol=1e-10, window_type="delta", mmax=int(np.ceil(3 * nev / s)))
    exact = lam_all[i1 - 1:i2]
    matched, legit, spurious = _classify(lam, exact, lam_all)
    assert spurious == 0 and matched >= nev - 2  # the window ends sit on eigenvalues
    assert res.max() < 1e-10 * 4.0


def test_polfed_xxz_exact_count(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(12, 5.0, 1)
    lam_all = np.linalg.eigvalsh(A.toarray())
    nrm = _norm2(lam_all)
    mid = np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1])))
    i_lo = mid - 15
    emin, emax = _window_with_gaps(lam_all, i_lo, i_lo + 29)
    smin, smax = O.gershgorin_bounds(A)
    lam, X, res = S.polfed(A, 30, 800, s=8, smin=smin, smax=smax, sigma=0.5 * (emin + emax),
                           emin=emin, emax=emax, window_type="step", mmax=14)
    assert lam.size == 30
    assert np.abs(np.sort(lam) - lam_all[i_lo:i_lo + 30]).max() <= 1e-12 * nrm
    assert res.max() <= 1e-10 * nrm
    r = np.linalg.norm(A @ X - X * lam, axis=0)
    assert np.abs(r - res).max() < 1e-12 * nrm
    assert np.abs(X.T @ X - np.eye(30)).max() < 1e-10


@pytest.mark.parametrize("degree,mmax,jackson", [(600, 12, True), (400, 16, False)])
def test_polfed_matches_oracle_same_start_block(lib_built, degree, mmax, jackson):
    """Also without Jackson damping (jackson=false, the undamped series: a sharper filter
    with Gibbs ripples), which converges here with a smaller degree and a larger basis."""
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(9, 16.5, 6)
    lam_all = np.linalg.eigvalsh(A.toarray())
    i0 = np.searchsorted(lam_all, 0.0) - 10
    emin, emax = _window_with_gaps(lam_all, i0, i0 + 19)
    smin, smax = O.gershgorin_bounds(A)
    kw = dict(s=8, smin=smin, smax=smax, sigma=0.0, emin=emin, emax=emax, window_type="step",
              mmax=mmax, tol=1e-10, jackson=jackson)
    lam_g, X_g, res_g = S.polfed(A, 20, degree, **kw)
    lam_o, X_o, res_o = O.polfed(A, 20, degree, **kw)
    nrm = _norm2(lam_all)
    assert lam_g.size == lam_o.size == 20
    assert np.abs(lam_g - lam_o).max() < 1e-12 * nrm
    assert np.abs(lam_g - lam_all[i0:i0 + 20]).max() < 1e-12 * nrm
    assert max(res_g.max(), res_o.max()) < 1e-10 * nrm


def test_polfed_device_callback_operator(lib_built):
    """A caller-supplied device matblock (here: the library's own SpMM on a device CSR
    copy, called from the callback on the solve's stream)."""
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    A = M.xxz_sz0(10, 2.0, 4)
    dev = S.SparseOperator(A)
    calls = []

    def matblock(X, Y, n, b, ld, stream):
        calls.append(b)
        return L.load().sma_spmm_dev(dev.handle, X, ld, Y, ld, b)

    matblock.device_block = True
    lam_all = np.linalg.eigvalsh(A.toarray())
    mid = len(lam_all) // 2
    emin, emax = _window_with_gaps(lam_all, mid - 5, mid + 4)
    smin, smax = O.gershgorin_bounds(A)
    lam, X, res = S.polfed(None, A.shape[0], 10, 500, matblock=matblock, s=4, smin=smin,
                           smax=smax, sigma=0.5 * (emin + emax), emin=emin, emax=emax, mmax=10)
    assert calls and lam.size == 10
    assert np.abs(np.sort(lam) - lam_all[mid - 5:mid + 5]).max() < 1e-12 * _norm2(lam_all)


def test_polfed_return_order_by_residual_when_not_converged(lib_built):
    """polfed.jl:1155-1156: below tol -> sorted by lambda; otherwise nev best by residual."""
    import sparse_matrix_algorithms_b200 as S

    A = M.anderson3d(8, 16.5, 5)
    smin, smax = O.gershgorin_bounds(A)
    lam, X, res = S.polfed(A, 10, 10, s=4, smin=smin, smax=smax, emin=-2.0, emax=2.0,
                           mmax=4, tol=1e-14)
    assert lam.size <= 10
    assert np.all(np.diff(res) >= 0)


def test_fp32_filter_solvers_run(lib_built):
    """Mixed precision: FP32 filter, FP64 orthogonalization and Rayleigh-Ritz."""
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(12, 5.0, 1)
    lam_all = np.linalg.eigvalsh(A.toarray())
    mid = np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1])))
    emin, emax = _window_with_gaps(lam_all, mid - 10, mid + 9)
    smin, smax = O.gershgorin_bounds(A)
    lam, X, res = S.polfed(A, 20, 800, s=8, smin=smin, smax=smax, sigma=0.5 * (emin + emax),
                           emin=emin, emax=emax, mmax=10, precision="fp32")
    assert lam.size == 20
    assert np.abs(np.sort(lam) - lam_all[mid - 10:mid + 10]).max() < 1e-5 * _norm2(lam_all)


# ---------------------------------------------------------------------- errors
def test_error_behaviour(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.lap1d(100)
    with pytest.raises(S.ArgumentError, match="symmetric"):
        S.chebyshev_poly_real_symm_sparse(sp.csr_matrix(np.triu(A.toarray())), 1.0, 2.0)
    with pytest.raises(S.ArgumentError, match="emin<emax"):
        S.chebyshev_poly_real_symm_sparse(A, 2.0, 1.0)
    with pytest.raises(S.ArgumentError, match="m0 must be positive"):
        S.chebyshev_poly_real_symm_sparse(A, 1.0, 2.0, m0=0)
    with pytest.raises(S.ArgumentError, match="not inside"):
        S.chebyshev_poly_real_symm_sparse(A, 1.0, 9.0, smin=0.0, smax=4.0)
    with pytest.raises(S.ArgumentError, match="requires spectral bounds"):
        S.polfed(A, 5, 10, s=4)
    with pytest.raises(S.ArgumentError, match="Unknown window"):
        S.polfed(A, 5, 10, s=4, smin=0.0, smax=4.0, window_type="hann")


def test_interval_outside_bounds_warns_then_raises(lib_built, capfd):
    """chebyshev_subspace_iteration.jl:683-689: @warn, then ArgumentError on the mapping."""
    import sparse_matrix_algorithms_b200 as S

    with pytest.raises(S.ArgumentError, match="not inside"):
        S.chebyshev_poly_real_symm_sparse(M.lap1d(200), 1.0, 1.2, smin=1.1, smax=4.0, m0=8,
                                          degree=10, maxiter=1)
    assert "not contained" in capfd.readouterr().err


def test_polfed_and_chebyshev_on_xxz_stencil_operator(lib_built):
    """Both solvers on the matrix-free XXZ stencil (no stored matrix) against the dense
    spectrum; bounds from GPU Lanczos on the stencil itself."""
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(12, 5.0, 1)
    lam_all = np.linalg.eigvalsh(A.toarray())
    nrm = _norm2(lam_all)
    mid = int(np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1]))))
    emin, emax = _window_with_gaps(lam_all, mid - 10, mid + 9)
    op = S.XXZOperator(12, 5.0, 1)
    smin, smax = S.lanczos_bounds(op, steps=60)
    assert smin <= lam_all[0] and smax >= lam_all[-1]
    lam, X, res = S.polfed(op, 20, 800, s=8, smin=smin, smax=smax, sigma=0.5 * (emin + emax),
                           emin=emin, emax=emax, mmax=10)
    assert lam.size == 20
    assert np.abs(np.sort(lam) - lam_all[mid - 10:mid + 10]).max() < 1e-12 * nrm
    assert res.max() < 1e-10 * nrm
    lam2, X2, res2 = S.chebyshev_poly_real_symm_sparse(op, emin, emax, smin=smin, smax=smax,
                                                       m0=40, degree=800, maxiter=10,
                                                       window_type="step")
    assert lam2.size == 20
    assert np.abs(lam2 - lam_all[mid - 10:mid + 10]).max() < 1e-12 * nrm


# ---------------------------------------------------------------------- bounds
@pytest.mark.parametrize("name", ["anderson_L20", "xxz_L18"])
def test_lanczos_bounds_enclose_spectrum_and_beat_gershgorin(lib_built, name):
    import sparse_matrix_algorithms_b200 as S
    from conftest import GOLDEN

    g = np.load(f"{GOLDEN}/{name}_spectrum.npz")
    lo_true, hi_true = float(g["lam_min"]), float(g["lam_max"])
    A = M.config_matrix(name)
    lo, hi = S.lanczos_bounds(A, steps=80)
    glo, ghi = O.gershgorin_bounds(A)
    assert lo <= lo_true and hi >= hi_true  # encloses the spectrum
    assert glo <= lo and hi <= ghi  # never looser than Gershgorin
    assert (hi - lo) < 0.95 * (ghi - glo)
    assert (hi - lo) < 1.01 * (hi_true - lo_true)


def test_lanczos_bounds_stencil_operator(lib_built):
    import sparse_matrix_algorithms_b200 as S

    lo, hi = S.lanczos_bounds(S.Lap1dOperator(3000), steps=120)
    ex = M.lap1d_exact_eigs(3000)
    assert lo <= ex[0] and hi >= ex[-1] and hi - lo < 4.01


# ---------------------------------------------------------------------- locking, precision
def _c1_reference():
    from conftest import GOLDEN

    g = np.load(f"{GOLDEN}/anderson_L20_spectrum.npz")
    c = g["central"]
    exact = c[(c >= -0.05) & (c <= 0.05)]
    return exact, max(abs(float(g["lam_min"])), abs(float(g["lam_max"])))


def test_chebyshev_locking_c1(lib_built):
    """Locking (lock=True): same eigenpairs as without, fewer filtered columns."""
    import sparse_matrix_algorithms_b200 as S

    exact, nrm = _c1_reference()
    A = S.SparseOperator(M.config_matrix("anderson_L20"))
    kw = dict(m0=64, degree=1500, maxiter=12, window_type="delta", sigma=0.0, tol=1e-11)
    st0, st1 = {}, {}
    lam0, X0, res0 = S.chebyshev_poly_real_symm_sparse(None, A.n, -0.05, 0.05, matblock=A,
                                                       smin=-14.25, smax=14.25, stats=st0, **kw)
    lam1, X1, res1 = S.chebyshev_poly_real_symm_sparse(None, A.n, -0.05, 0.05, matblock=A,
                                                       smin=-14.25, smax=14.25, lock=True,
                                                       stats=st1, **kw)
    for lam, res in [(lam0, res0), (lam1, res1)]:
        assert lam.size == exact.size
        assert np.abs(lam - exact).max() <= 1e-12 * nrm
        assert res.max() <= 1e-10 * nrm
    assert st1["locked"] > 0
    assert st1["spmm_columns"] < st0["spmm_columns"]
    Ad = M.config_matrix("anderson_L20")
    assert np.abs(np.linalg.norm(Ad @ X1 - X1 * lam1, axis=0) - res1).max() < 1e-12
    assert np.abs(X1.T @ X1 - np.eye(lam1.size)).max() < 1e-10


def test_chebyshev_mixed_precision_c1(lib_built):
    """MIXED: FP32 filter first, FP64 for the final iterations; FP64-quality pairs."""
    import sparse_matrix_algorithms_b200 as S

    exact, nrm = _c1_reference()
    A = S.SparseOperator(M.config_matrix("anderson_L20"))
    st = {}
    lam, X, res = S.chebyshev_poly_real_symm_sparse(
        None, A.n, -0.05, 0.05, matblock=A, smin=-14.25, smax=14.25, m0=64, degree=1500,
        maxiter=16, window_type="delta", sigma=0.0, precision="mixed", stats=st)
    assert st["fp32_filter_calls"] >= 1
    assert lam.size == exact.size
    assert np.abs(lam - exact).max() <= 1e-12 * nrm
    assert res.max() <= 1e-10 * nrm


def test_polfed_mixed_precision_xxz(lib_built):
    """POLFED with an FP32-filtered basis and FP64 polishing."""
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(12, 5.0, 1)
    lam_all = np.linalg.eigvalsh(A.toarray())
    nrm = _norm2(lam_all)
    mid = int(np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1]))))
    emin, emax = _window_with_gaps(lam_all, mid - 10, mid + 9)
    smin, smax = O.gershgorin_bounds(A)
    st = {}
    lam, X, res = S.polfed(A, 20, 800, s=8, smin=smin, smax=smax, sigma=0.5 * (emin + emax),
                           emin=emin, emax=emax, mmax=10, precision="mixed", stats=st)
    assert st["fp32_filter_calls"] >= 1
    assert lam.size == 20
    assert np.abs(np.sort(lam) - lam_all[mid - 10:mid + 10]).max() <= 1e-12 * nrm
    assert res.max() <= 1e-10 * nrm


@pytest.mark.parametrize("env", [{"SMA_POLISH_FILTER_GUARDS": "1"},
                                 {"SMA_POLISH_REFINE": "1"},
                                 {"SMA_POLISH_FILTER": "step", "SMA_POLISH_GUARDS": "2"}])
def test_polfed_mixed_polish_variants(lib_built, monkeypatch, env):
    """The polish's alternative settings (filtered guards with a Rayleigh-Ritz first, the
    refinement kept, an undamped step polynomial over the guards' span with fewer guards)
    reach the same pairs as the default: the exact count, |dlambda| <= 1e-12 ||A||, relative
    residual <= 1e-10, and residuals that match the returned vectors."""
    import sparse_matrix_algorithms_b200 as S

    for k, v in env.items():
        monkeypatch.setenv(k, v)
    A = M.xxz_sz0(12, 5.0, 1)
    lam_all = np.linalg.eigvalsh(A.toarray())
    nrm = _norm2(lam_all)
    mid = int(np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1]))))
    emin, emax = _window_with_gaps(lam_all, mid - 10, mid + 9)
    smin, smax = O.gershgorin_bounds(A)
    st = {}
    lam, X, res = S.polfed(A, 20, 800, s=8, smin=smin, smax=smax, sigma=0.5 * (emin + emax),
                           emin=emin, emax=emax, mmax=10, precision="mixed", stats=st)
    assert st["polish_iterations"] >= 1
    assert lam.size == 20
    assert np.abs(np.sort(lam) - lam_all[mid - 10:mid + 10]).max() <= 1e-12 * nrm
    assert res.max() <= 1e-10 * nrm
    r = np.linalg.norm(A @ X - X * lam, axis=0)
    assert np.abs(r - res).max() <= 1e-12 * nrm


def test_filter_graph_replay_is_bit_identical(lib_built, monkeypatch):
    """POLFED calls the same filter once per block: from the second call the recurrence is
    replayed from a CUDA graph.  A context with graphs off gives bit-identical results."""
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(14, 5.0, 1)
    lam_all = np.linalg.eigvalsh(A.toarray())
    mid = int(np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1]))))
    emin, emax = _window_with_gaps(lam_all, mid - 15, mid + 14)
    smin, smax = O.gershgorin_bounds(A)
    kw = dict(s=16, smin=smin, smax=smax, sigma=0.5 * (emin + emax), emin=emin, emax=emax,
              mmax=8, window_type="delta")
    st = {}
    lam, X, res = S.polfed(S.SparseOperator(A), 30, 900, stats=st, **kw)
    assert st["graph_replays"] == 7
    monkeypatch.setenv("SMA_FILTER_GRAPHS", "0")
    ctx = S.Context(0)
    st0 = {}
    lam0, X0, res0 = S.polfed(S.SparseOperator(A, ctx), 30, 900, stats=st0, **kw)
    assert st0["graph_replays"] == 0
    np.testing.assert_array_equal(lam, lam0)
    np.testing.assert_array_equal(res, res0)
    np.testing.assert_array_equal(X, X0)
    # the same kernels, plus the staging copies in and out of each replay
    assert st["kernel_launches"] == st0["kernel_launches"] + 2 * 7
