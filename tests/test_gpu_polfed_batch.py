"""Batched POLFED (sma_polfed_batch_solve): several windows of one matrix, every block step
filtering all windows' blocks in one segmented recurrence.

* FP64: each window's eigenpairs are bit-identical to the single-window POLFED solve with
  the same (nev, degree, mmax, seed) -- the segmented filter reproduces the single filter
  bit for bit and the rest of a window's solve is the same code.
* Against the dense spectrum (XXZ L=14, n=3432): every window's count exact, |dlambda| <=
  1e-12 ||A||, relative residual <= 1e-10, in FP64 and in MIXED precision (FP32 basis
  filter, FP64 polish), for windows of uneven counts and degrees (the reference's checks,
  chebyshev_subspace_iteration.jl:905-979; polfed.jl:1148-1157 for the return order).
"""
import numpy as np
import pytest

import sma_oracle as O
from sparse_matrix_algorithms_b200 import matrices as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def xxz14(lib_built):
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(14, 5.0, 1)
    lam_all = np.linalg.eigvalsh(A.toarray())
    smin, smax = O.gershgorin_bounds(A)
    return A, S.SparseOperator(A), lam_all, smin, smax


def _windows(lam_all, counts, start):
    """Contiguous windows holding exactly `counts` eigenvalues each, ends at mid-gaps."""
    out, i = [], start
    for c in counts:
        out.append((0.5 * (lam_all[i - 1] + lam_all[i]), 0.5 * (lam_all[i + c - 1] + lam_all[i + c]), i, c))
        i += c
    return out


def _plan(lam_all, smin, smax, wins, s):
    d = 0.5 * (smax - smin)
    nev = [c + 4 for *_, c in wins]
    deg = [int(np.ceil(10 * d / (b - a))) for a, b, *_ in wins]
    mmax = [int(np.ceil(4.0 * c / s)) + 2 for *_, c in wins]
    return nev, deg, mmax


def test_batched_windows_equal_single_window_solves(xxz14):
    import sparse_matrix_algorithms_b200 as S

    A, op, lam_all, smin, smax = xxz14
    mid = int(np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1]))))
    wins = _windows(lam_all, [12, 30, 20], mid - 30)
    s = 8
    nev, deg, mmax = _plan(lam_all, smin, smax, wins, s)
    kw = dict(s=s, smin=smin, smax=smax, window_type="step", seed=5)
    st = {}
    lam_b, X_b, res_b, win_b = S.polfed_windows(op, [w[:2] for w in wins], nev, deg, mmax,
                                                stats=st, **kw)
    assert st["graph_replays"] > 0  # the batched recurrence was replayed from a graph
    for w, (a, b, i0, c) in enumerate(wins):
        lam_s, X_s, res_s = S.polfed(op, nev[w], deg[w], emin=a, emax=b, sigma=0.5 * (a + b),
                                     mmax=mmax[w], s=s, smin=smin, smax=smax,
                                     window_type="step", seed=5 + w)
        sel = win_b == w
        assert np.array_equal(lam_b[sel], lam_s)
        assert np.array_equal(res_b[sel], res_s)
        assert np.array_equal(X_b[:, sel], X_s)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_windows_against_dense_spectrum(xxz14, precision):
    import sparse_matrix_algorithms_b200 as S

    A, op, lam_all, smin, smax = xxz14
    nrm = max(abs(lam_all[0]), abs(lam_all[-1]))
    mid = int(np.argmin(np.abs(lam_all - 0.5 * (lam_all[0] + lam_all[-1]))))
    wins = _windows(lam_all, [8, 40, 16, 25, 10], mid - 50)
    s = 8
    nev, deg, mmax = _plan(lam_all, smin, smax, wins, s)
    st = {}
    lam, X, res, win = S.polfed_windows(op, [w[:2] for w in wins], nev, deg, mmax, s=s,
                                        smin=smin, smax=smax, window_type="step",
                                        precision=precision, stats=st)
    for w, (a, b, i0, c) in enumerate(wins):
        sel = win == w
        inside = sel & (lam >= a) & (lam <= b)
        assert int(inside.sum()) == c, (w, int(inside.sum()), c)
        got = np.sort(lam[inside])
        assert np.abs(got - lam_all[i0:i0 + c]).max() <= 1e-12 * nrm
        assert res[inside].max() <= 1e-10 * nrm
    r = np.linalg.norm(A @ X - X * lam, axis=0)
    assert np.abs(r - res).max() <= 1e-12 * nrm
    if precision == "mixed":
        assert st["fp32_filter_calls"] > 0 and st["polish_iterations"] >= 1
