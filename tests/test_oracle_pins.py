"""Pins of the CPU oracle against the reference's own known answers.

The reference has no stored fixtures; its tests (script blocks at the end of each
file) compare against the analytic 1D-Laplacian spectrum and print results.  These
tests pin the oracle to those known answers, to the algebraic identities the
reference's formulas imply, and to the reference's published 1D-Laplacian runs
(``tests/golden/published_runs.json``).
"""
import json
import math
import os

import numpy as np
import pytest
import scipy.sparse as sp

import sma_oracle as O
from sparse_matrix_algorithms_b200 import matrices as M

from conftest import GOLDEN


def test_jackson_kernel_first_coefficient_is_one():
    # g_0 = 1/(K+2) + (K+1)/(K+2) = 1  (chebyshev_subspace_iteration.jl:382)
    for K in [1, 2, 7, 64, 500, 3500]:
        g = O.jackson_kernel(K)
        assert len(g) == K + 1
        assert abs(g[0] - 1.0) < 4e-16
        assert np.all(np.diff(g) <= 1e-15)  # monotone damping
    assert O.jackson_kernel(0).tolist() == [1.0]


def test_full_interval_window_is_identity():
    # cheb_window_coeffs(-1, 1, K): c_0 = 1, c_k = 2 sin(k pi)/(k pi) ~ 0
    for K in [0, 1, 10, 200]:
        c = O.cheb_window_coeffs(-1.0, 1.0, K, jackson=False)
        assert c[0] == 1.0
        assert np.abs(c[1:]).max(initial=0.0) < 1e-15
    A = M.lap1d(300)
    Q = M.splitmix_normal(3, 300, 5)
    c = O.cheb_window_coeffs(-1.0, 1.0, 40, jackson=True)
    Y = O.apply_poly_block(A, Q, c, 0.0, 4.0)
    assert np.abs(Y - Q).max() < 1e-12 * np.abs(Q).max()


@pytest.mark.parametrize("window", ["step", "delta", "smooth"])
def test_clenshaw_on_diagonal_matrix_is_pointwise_series(window):
    n, K = 400, 57
    rng = np.random.default_rng(1)
    d = np.sort(rng.uniform(-3.0, 5.0, n))
    A = sp.diags(d).tocsr()
    smin, smax = -3.5, 5.5
    c = O.build_coeffs(K, smin, smax, 0.7, 0.1, 1.3, window, True)
    x = (d - 0.5 * (smin + smax)) / (0.5 * (smax - smin))
    pval = np.polynomial.chebyshev.chebval(x, c)
    Q = M.splitmix_normal(11, n, 3)
    for impl in ["c", "numpy"]:
        Y = O.apply_poly_block(A, Q, c, smin, smax, impl=impl)
        assert np.abs(Y - pval[:, None] * Q).max() < 1e-12 * np.abs(Q).max()


def test_c_and_numpy_filters_agree_bitwise():
    A = M.anderson3d(6, 16.5, 5)
    Q = M.splitmix_normal(2, A.shape[0], 7)
    c = O.build_coeffs(90, -15.0, 15.0, 0.0, -0.5, 0.5, "step", True)
    Y1 = O.apply_poly_block(A, Q, c, -15.0, 15.0, impl="c")
    Y2 = O.apply_poly_block(A, Q, c, -15.0, 15.0, impl="numpy")
    assert np.array_equal(Y1, Y2)


def test_gershgorin_matches_definition():
    A = M.anderson3d(5, 16.5, 0)
    lo, hi = O.gershgorin_bounds(A)
    D = A.toarray()
    r = np.abs(D).sum(1) - np.abs(np.diag(D))
    assert lo == np.min(np.diag(D) - r) and hi == np.max(np.diag(D) + r)
    ev = np.linalg.eigvalsh(D)
    assert lo <= ev[0] and ev[-1] <= hi


def test_lap1d_windows_follow_reference():
    lam, i1, i2, emin, emax, sigma = M.lap1d_target_window(1000, 100)
    assert (i1, i2) == (450, 549)  # mid=500, i1 = 500 - fld(100, 2)
    assert emin == lam[449] and emax == lam[548]
    emin2, emax2, sig2, lref, (j1, j2) = M.lap1d_interval_by_count(1000, 100)
    assert (j1, j2) == (450, 549) and emin2 == lam[447] and emax2 == lam[550]
    assert np.array_equal(lref, lam[449:549])


def _classify(lam_got, lam_ref, lam_all, tol=1e-8):
    """matched / legit-extra / spurious counts (chebyshev_subspace_iteration.jl:918-979)."""
    got = np.sort(lam_got)
    matched = sum(np.min(np.abs(got - r)) <= tol for r in lam_ref) if got.size else 0
    legit = sum(np.min(np.abs(lam_all - g)) <= tol for g in got)
    return matched, legit, got.size - legit


def test_oracle_chebyshev_lap1d_known_answer():
    n, nev = 2000, 40
    emin, emax, sigma, lref, _ = M.lap1d_interval_by_count(n, nev)
    lam, X, res = O.chebyshev_poly_real_symm_sparse(
        M.lap1d(n), emin, emax, smin=0.0, smax=4.0, sigma=sigma, m0=2 * nev, degree=128,
        maxiter=10, tol=1e-8, window_type="delta")
    matched, legit, spurious = _classify(lam, lref, M.lap1d_exact_eigs(n))
    assert matched == nev and spurious == 0
    assert res.max() < 1e-8
    assert np.abs(np.linalg.norm(X, axis=0) - 1).max() < 1e-12


def test_oracle_polfed_lap1d_known_answer():
    n, nev = 3000, 60
    lam_all, i1, i2, emin, emax, sigma = M.lap1d_target_window(n, nev)
    # a window with margins so that the count is well defined
    gap = lam_all[i1 - 1] - lam_all[i1 - 2]
    lam, X, res = O.polfed(M.lap1d(n), nev, 200, s=16, smin=0.0, smax=4.0, sigma=sigma,
                           emin=emin - gap / 2, emax=emax + gap / 2, mmax=16,
                           window_type="smooth", tol=1e-10)
    assert lam.size == nev
    assert np.abs(np.sort(lam) - lam_all[i1 - 1:i2]).max() < 1e-12 * 4.0
    assert res.max() < 1e-10 * 4.0


def test_published_runs_fixture_is_consistent():
    """The reference's published 1D-Laplacian runs, as committed golden data."""
    with open(os.path.join(GOLDEN, "published_runs.json")) as f:
        runs = json.load(f)
    assert {r["solver"] for r in runs["runs"]} == {"chebyshev", "polfed"}
    for r in runs["runs"]:
        assert r["found"] <= r["nev"] + 10
        if r["solver"] == "polfed":
            assert r["mmax"] == math.ceil(r["b"] * r["nev"] / r["s"])


@pytest.mark.slow
def test_oracle_reproduces_published_polfed_n10000():
    """polfed.jl:1279-1288: n=10000, nev=1000, s=64, degree=32, b=5 (mmax=79)
    -> inside=1000, maxres 3.1e-14.  The harness window ends sit exactly on eigenvalues
    (polfed.jl:1223-1233), so the two boundary pairs fall inside or outside by rounding;
    the reference's own runs report 998-1000.  The oracle's runs (make_golden.py) are
    stored in tests/golden/oracle_published_polfed_n10000.json."""
    path = os.path.join(GOLDEN, "oracle_published_polfed_n10000.json")
    with open(path) as f:
        g = json.load(f)
    pub = json.load(open(os.path.join(GOLDEN, "published_runs.json")))["runs"][1]
    assert pub["n"] == 10000 and pub["found"] == 1000
    for run in g["runs"].values():
        assert 998 <= run["inside"] <= 1000
        assert run["matched"] >= 998 and run["spurious"] == 0
        assert run["maxres"] < 10 * pub["maxres"]
        assert run["max_abs_err_vs_exact"] < 1e-12
