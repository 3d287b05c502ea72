"""ORACLE -- test infrastructure only, never part of the product.

A CPU FP64 restatement of the reference's two solve-free interior eigensolvers,
written function by function from the Julia sources so that the CUDA library can be
checked against it on identical inputs.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` import this module.

Citations are ``file:line`` into MathiasTensor/sparse_matrix_algorithms:
``chebyshev_subspace_iteration.jl`` (below: *cheb*) and ``polfed.jl``.

Differences from the reference that do not change results
---------------------------------------------------------
* ``randn`` (Julia's Xoshiro stream) is not reproducible outside Julia; the random
  start block comes from the documented SplitMix64/Box-Muller generator
  (``sparse_matrix_algorithms_b200.matrices.splitmix_normal``), the same formula the
  CUDA library evaluates.  Parity is compared on converged eigenpairs.
* Householder QR and the dense symmetric eigensolves go through numpy's LAPACK
  (``dgeqrf``/``dorgqr``, ``dsyevd``) where Julia's ``qr!``/``eigen`` call
  ``geqrt``/``syevr``: same factorizations, rounding-level differences, eigenvector
  signs free.
* The block Clenshaw filter has two implementations: :func:`apply_poly_block_numpy`
  (scipy CSR products) and the C restatement ``clenshaw_ref.c`` (same arithmetic order
  as Julia's CSC ``mul!``), selected by ``impl``.

Pinning: ``tests/test_oracle_pins.py`` checks this module against the reference's
known answers -- the analytic 1D-Laplacian spectrum, ``jackson_kernel(K)[1] == 1``,
the identity filter ``cheb_window_coeffs(-1, 1, K)``, Clenshaw on a diagonal matrix --
and against the reference's published 1D-Laplacian runs (golden fixtures under
``tests/golden/``).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import sys
from typing import Callable, List, Optional, Tuple

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))
from sparse_matrix_algorithms_b200.matrices import splitmix_normal  # noqa: E402

# ======================================================================================
# C restatement loader
# ======================================================================================

_LIB = None


def build_c_oracle() -> str:
    """Compile ``clenshaw_ref.c`` (``make -C oracle``) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "_build", "liboracle.so")


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liboracle.so")
        src = os.path.join(_HERE, "clenshaw_ref.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build_c_oracle()
        lib = ctypes.CDLL(path)
        i64, dp = ctypes.c_int64, ctypes.c_void_p
        lib.oracle_apply_poly_block.argtypes = [i64, i64, dp, dp, dp, dp, dp, dp, i64,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_int]
        lib.oracle_spmm.argtypes = [i64, i64, dp, dp, dp, dp, dp, ctypes.c_int]
        _LIB = lib
    return _LIB


def _csc_arrays(A):
    """0-based int64 CSC arrays of a (symmetric) sparse matrix."""
    C = sp.csc_matrix(A)
    C.sort_indices()
    return (np.ascontiguousarray(C.indptr, dtype=np.int64),
            np.ascontiguousarray(C.indices, dtype=np.int64),
            np.ascontiguousarray(C.data, dtype=np.float64))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# ======================================================================================
# operators
# ======================================================================================

class MatrixFreeRealSymOp:
    """Matrix-free operator (cheb:151-167, polfed:148-165) for the oracle.

    ``matvec(y, x)`` writes A x into y; optional ``matblock(Y, X)`` writes A X into Y.
    """

    def __init__(self, n: int, matvec: Callable, matblock: Optional[Callable] = None):
        self.n = n
        self.matvec = matvec
        self.matblock = matblock
        self.shape = (n, n)


def apply_A_block(Y: np.ndarray, A, X: np.ndarray, impl: str = "c", nthreads: int = 0) -> np.ndarray:
    """Y <- A X (cheb:186-197, polfed:196-219)."""
    if isinstance(A, MatrixFreeRealSymOp):
        if A.matblock is not None:
            A.matblock(Y, X)
        else:
            for j in range(X.shape[1]):
                y = np.empty(X.shape[0])
                A.matvec(y, X[:, j].copy())
                Y[:, j] = y
        return Y
    if impl == "c" and X.shape[1] > 0:
        colptr, rowval, nzval = _cached_csc(A)
        Xf = np.asfortranarray(X, dtype=np.float64)
        Yf = np.empty_like(Xf, order="F")
        _lib().oracle_spmm(X.shape[0], X.shape[1], _ptr(colptr), _ptr(rowval), _ptr(nzval),
                           _ptr(Xf), _ptr(Yf), nthreads)
        Y[...] = Yf
        return Y
    Y[...] = A @ X
    return Y


_CSC_CACHE: dict = {}


def _cached_csc(A):
    key = id(A)
    hit = _CSC_CACHE.get(key)
    if hit is not None and hit[0] is A:
        return hit[1]
    arrs = _csc_arrays(A)
    _CSC_CACHE.clear()
    _CSC_CACHE[key] = (A, arrs)
    return arrs


# ======================================================================================
# spectral bounds and filter coefficients
# ======================================================================================

def gershgorin_bounds(A) -> Tuple[float, float]:
    """(min_i(a_ii - r_i), max_i(a_ii + r_i)), r_i = sum_{j!=i}|a_ij| (cheb:351-367)."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    if A.shape[1] != n:
        raise ValueError("A must be square")
    d = A.diagonal()
    absA = abs(A)
    r = np.asarray(absA.sum(axis=1)).ravel() - np.abs(d)
    return float(np.min(d - r)), float(np.max(d + r))


def jackson_kernel(K: int) -> np.ndarray:
    """Jackson damping g_0..g_K (cheb:376-387)."""
    if K <= 0:
        return np.array([1.0])
    a = math.pi / (K + 2)
    sa = math.sin(a)
    g = np.empty(K + 1)
    for k in range(K + 1):
        g[k] = math.sin((k + 1) * a) / ((K + 2) * sa) + (1 - (k + 1) / (K + 2)) * math.cos(k * a)
    return g


def cheb_delta_coeffs(sigma_hat: float, K: int, jackson: bool = True) -> np.ndarray:
    """Delta-peak coefficients (cheb:400-414)."""
    c = np.zeros(K + 1)
    th = math.acos(min(max(sigma_hat, -1.0), 1.0))
    c[0] = 1 / math.pi
    for k in range(1, K + 1):
        c[k] = 2 * math.cos(k * th) / math.pi
    if jackson:
        c *= jackson_kernel(K)
    return c


def cheb_window_coeffs(a: float, b: float, K: int, jackson: bool = True) -> np.ndarray:
    """Step-indicator coefficients of [a, b] (cheb:430-447)."""
    aa = max(-1.0, min(1.0, a))
    bb = max(-1.0, min(1.0, b))
    if aa > bb:
        aa, bb = bb, aa
    al = math.acos(bb)
    be = math.acos(aa)
    c = np.zeros(K + 1)
    c[0] = (be - al) / math.pi
    for k in range(1, K + 1):
        c[k] = 2 * (math.sin(k * be) - math.sin(k * al)) / (k * math.pi)
    if jackson:
        c *= jackson_kernel(K)
    return c


def cheb_smooth_window_coeffs(a: float, b: float, K: int, jackson: bool = True,
                              nsamp: int = 4096, delta: float = 0.02) -> np.ndarray:
    """tanh-ramp window by trapezoid quadrature in theta (cheb:465-489)."""
    aa = max(-1.0, min(1.0, a))
    bb = max(-1.0, min(1.0, b))
    if aa > bb:
        aa, bb = bb, aa
    w = math.pi / (nsamp - 1)
    th = np.arange(nsamp) * w
    xi = np.cos(th)
    fi = 0.5 * (1 + np.tanh((xi - aa) / delta)) * 0.5 * (1 - np.tanh((xi - bb) / delta))
    wt = np.ones(nsamp)
    wt[0] = wt[-1] = 0.5
    f = wt * fi
    c = np.empty(K + 1)
    for k in range(K + 1):
        s = float(np.dot(f, np.cos(k * th)))
        c[k] = (1 / math.pi if k == 0 else 2 / math.pi) * w * s
    if jackson:
        c *= jackson_kernel(K)
    return c


def build_coeffs(degree, smin, smax, sigma, emin, emax, window_type="step", jackson=True):
    """Map to [-1, 1] and dispatch on the window type (polfed:404-414, cheb:685-700)."""
    c = 0.5 * (smin + smax)
    d = 0.5 * (smax - smin)
    sh = (sigma - c) / d
    a = (emin - c) / d
    b = (emax - c) / d
    if window_type == "step":
        return cheb_window_coeffs(a, b, degree, jackson)
    if window_type == "delta":
        return cheb_delta_coeffs(sh, degree, jackson)
    if window_type == "smooth":
        return cheb_smooth_window_coeffs(a, b, degree, jackson)
    raise ValueError(f"Unknown window type: {window_type}")


# ======================================================================================
# block Clenshaw filter
# ======================================================================================

def apply_poly_block_numpy(A, Q: np.ndarray, coeffs: np.ndarray, smin: float, smax: float) -> np.ndarray:
    """Y = p(A_hat) Q by block Clenshaw (cheb:554-591 / polfed:464-501)."""
    K = len(coeffs) - 1
    c = 0.5 * (smin + smax)
    invd = 2.0 / (smax - smin)
    alpha = 2.0 * invd
    beta = -2.0 * c * invd
    B1 = np.zeros_like(Q)
    B2 = np.zeros_like(Q)
    AX = np.empty_like(Q)
    for k in range(K + 1, 1, -1):
        apply_A_block(AX, A, B1, impl="numpy")
        ck = coeffs[k - 1]
        TMP = ck * Q + alpha * AX + beta * B1 - B2
        B1, B2 = TMP, B1
    apply_A_block(AX, A, B1, impl="numpy")
    return coeffs[0] * Q + invd * AX - c * invd * B1 - B2


def apply_poly_block(A, Q: np.ndarray, coeffs: np.ndarray, smin: float, smax: float,
                     impl: str = "c", nthreads: int = 0) -> np.ndarray:
    """Block Clenshaw filter; ``impl="c"`` runs ``clenshaw_ref.c`` (sparse A only)."""
    if impl != "c" or isinstance(A, MatrixFreeRealSymOp) or Q.shape[1] == 0:
        return apply_poly_block_numpy(A, Q, coeffs, smin, smax)
    colptr, rowval, nzval = _cached_csc(A)
    Qf = np.asfortranarray(Q, dtype=np.float64)
    Y = np.empty_like(Qf, order="F")
    cf = np.ascontiguousarray(coeffs, dtype=np.float64)
    rc = _lib().oracle_apply_poly_block(Q.shape[0], Q.shape[1], _ptr(colptr), _ptr(rowval),
                                        _ptr(nzval), _ptr(Qf), _ptr(Y), _ptr(cf), len(cf) - 1,
                                        float(smin), float(smax), nthreads)
    if rc != 0:
        raise RuntimeError("oracle_apply_poly_block failed")
    return Y


# ======================================================================================
# orthogonalization
# ======================================================================================

def thin_orth(Qc: np.ndarray) -> np.ndarray:
    """Householder QR, keep the thin Q (cheb:223-231)."""
    Q, _ = np.linalg.qr(Qc, mode="reduced")
    return Q


def _truncated_qr(W: np.ndarray, rtol: float):
    n, m = W.shape
    if min(n, m) == 0:
        return np.empty((n, 0)), np.empty((0, m))
    Q, R = np.linalg.qr(W, mode="reduced")
    k = min(R.shape)
    dr = np.abs(np.diag(R[:k, :k]))
    r0 = dr.max()
    if r0 == 0:
        return np.empty((n, 0)), np.empty((0, m))
    r = int(np.count_nonzero(dr > rtol * r0))
    if r == 0:
        return np.empty((n, 0)), np.empty((0, m))
    return Q[:, :r].copy(), R[:r, :m].copy()


def orth_block(Q: np.ndarray, rtol: float = 1e-12) -> np.ndarray:
    """Rank-truncating QR: keep the first count(|R_ii| > rtol*max|R_ii|) columns
    (cheb:268-279, polfed:561-594)."""
    return _truncated_qr(Q, rtol)[0]


def orth_against(W: np.ndarray, Q: np.ndarray) -> np.ndarray:
    """W <- W - Q(Q^T W) (cheb:248-252, polfed:605-609)."""
    if Q.shape[1] == 0:
        return W
    W -= Q @ (Q.T @ W)
    return W


def reorth_full(W: np.ndarray, Qhist: List[np.ndarray], Qcur: np.ndarray, passes: int = 1) -> np.ndarray:
    """Project against every stored block, then the current one (polfed:623-631)."""
    for _ in range(passes):
        for Q in Qhist:
            orth_against(W, Q)
        orth_against(W, Qcur)
    return W


def block_qr_factor(W: np.ndarray, rtol: float = 1e-12):
    """W ~ Q B with rank truncation (polfed:644-685)."""
    return _truncated_qr(W, rtol)


# ======================================================================================
# Rayleigh quotients, residuals, refinement
# ======================================================================================

def residuals(A, X: np.ndarray, lam: np.ndarray, impl: str = "c") -> np.ndarray:
    """res_j = ||A x_j - lam_j x_j|| (cheb:311-344)."""
    AX = np.empty_like(X)
    apply_A_block(AX, A, X, impl=impl)
    return np.sqrt(np.sum((AX - X * lam[None, :]) ** 2, axis=0))


def rayleigh(A, X: np.ndarray, impl: str = "c"):
    """lam_j = x_j^T A x_j, res_j = ||A x_j - lam_j x_j|| (polfed:791-830)."""
    AX = np.empty_like(X)
    apply_A_block(AX, A, X, impl=impl)
    lam = np.einsum("ij,ij->j", X, AX)
    res = np.sqrt(np.sum((AX - X * lam[None, :]) ** 2, axis=0))
    return lam, res


def refine_original_rr(A, X: np.ndarray, rtol: float = 1e-12, impl: str = "c"):
    """Original-space Rayleigh-Ritz on span(X), sorted by lambda (polfed:837-880)."""
    Q = orth_block(X.copy(), rtol)
    k = Q.shape[1]
    if k == 0:
        return np.empty(0), np.empty((X.shape[0], 0)), np.empty(0)
    AQ = np.empty_like(Q)
    apply_A_block(AQ, A, Q, impl=impl)
    H = 0.5 * (Q.T @ AQ + AQ.T @ Q)
    _, U = np.linalg.eigh(H)
    Y = Q @ U
    lam, res = rayleigh(A, Y, impl=impl)
    p = np.argsort(lam, kind="stable")
    return lam[p], Y[:, p], res[p]


# ======================================================================================
# Chebyshev filtered subspace iteration
# ======================================================================================

def chebyshev_poly_real_symm_sparse(A, emin: float, emax: float, *, smin=None, smax=None,
                                    sigma: float = 0.0, m0: int = 200, degree: int = 80,
                                    maxiter: int = 8, tol: float = 1e-10, res_gate: float = 1e-6,
                                    jackson: bool = True, debug: bool = False,
                                    two_hit: bool = True, seed: int = 1,
                                    window_type: str = "step", matrix_free: Optional[bool] = None,
                                    impl: str = "c", Q0: Optional[np.ndarray] = None,
                                    history: Optional[list] = None):
    """Chebyshev-filtered subspace iteration.

    Sparse overload (cheb:667-757): runs all ``maxiter`` iterations.  Matrix-free
    overload (cheb:771-848, selected when ``A`` is a :class:`MatrixFreeRealSymOp` or
    ``matrix_free=True``): stops on the ``two_hit`` rule.  Returns
    ``(lam, X, res)`` sorted by lambda, residuals absolute.
    """
    mf = isinstance(A, MatrixFreeRealSymOp) if matrix_free is None else matrix_free
    n = A.shape[0]
    if not mf:
        if A.shape[1] != n:
            raise ValueError("A must be square")
        if (abs(sp.csr_matrix(A) - sp.csr_matrix(A).T)).nnz != 0:
            raise ValueError("Chebyshev filtered solver requires a real symmetric matrix")
        if not emin < emax:
            raise ValueError("need emin<emax")
        if m0 <= 0:
            raise ValueError("m0 must be positive")
        if degree < 0:
            raise ValueError("degree must be nonnegative")
    m0 = min(m0, n)
    if smin is None or smax is None:
        smin_, smax_ = gershgorin_bounds(A)
    else:
        smin_, smax_ = smin, smax
    c = 0.5 * (smin_ + smax_)
    d = 0.5 * (smax_ - smin_)
    a = (emin - c) / d
    b = (emax - c) / d
    if not (-1.0 <= a < b <= 1.0):
        raise ValueError(f"mapped interval [{a},{b}] not inside [-1,1]")
    coeffs = build_coeffs(degree, smin_, smax_, sigma, emin, emax, window_type, jackson)
    Q = splitmix_normal(seed, n, m0) if Q0 is None else np.array(Q0, dtype=np.float64, order="F")
    prev_ok = False
    lam = res = X = None
    for it in range(1, maxiter + 1):
        Y = apply_poly_block(A, Q, coeffs, smin_, smax_, impl=impl)
        Q = thin_orth(Y)
        R = np.empty_like(Q)
        apply_A_block(R, A, Q, impl=impl)
        Aq = Q.T @ R
        # Julia's Symmetric(Aq) reads the upper triangle
        Aq = np.triu(Aq) + np.triu(Aq, 1).T
        lam, Xq = np.linalg.eigh(Aq)
        X = Q @ Xq
        res = residuals(A, X, lam, impl=impl)
        inside = (lam >= emin) & (lam <= emax) & (res < res_gate)
        maxres = float(res[inside].max()) if inside.any() else math.inf
        if history is not None:
            history.append((it, int(inside.sum()), maxres))
        if debug:
            print(f"it={it} inside={int(inside.sum())} maxres={maxres:.3e}")
        if mf:
            ok = bool(inside.any()) and maxres < tol
            if two_hit:
                if ok and (it == 1 or prev_ok):
                    break
                prev_ok = ok
            elif ok:
                break
    sel = (lam >= emin) & (lam <= emax) & (res < max(res_gate, 10 * tol))
    idx = np.nonzero(sel)[0]
    if idx.size == 0:
        return np.empty(0), np.empty((n, 0)), np.empty(0)
    p = np.argsort(lam[idx], kind="stable")
    idx = idx[p]
    return lam[idx].copy(), X[:, idx].copy(), res[idx].copy()


# ======================================================================================
# POLFED
# ======================================================================================

def assemble_T(Ablocks: List[np.ndarray], Bblocks: List[np.ndarray]) -> np.ndarray:
    """Dense symmetric block tridiagonal T (polfed:701-754)."""
    dims = [a.shape[0] for a in Ablocks]
    N = sum(dims)
    T = np.zeros((N, N))
    o = 0
    for j, Aj in enumerate(Ablocks):
        r = dims[j]
        T[o:o + r, o:o + r] = Aj
        if j < len(Ablocks) - 1:
            B = Bblocks[j]
            T[o + r:o + r + B.shape[0], o:o + r] = B
            T[o:o + r, o + r:o + r + B.shape[0]] = B.T
        o += r
    return T


def build_X(Qhist: List[np.ndarray], U: np.ndarray) -> np.ndarray:
    """X = sum_j Q_j U[rows of block j, :] (polfed:767-776)."""
    X = np.zeros((Qhist[0].shape[0], U.shape[1]))
    o = 0
    for Q in Qhist:
        r = Q.shape[1]
        X += Q @ U[o:o + r, :]
        o += r
    return X


def build_full_basis(A, Q1, coeffs, smin, smax, mmax, rtol=1e-12, reorth_passes=1, impl="c"):
    """Block Lanczos on p(A_hat) with full reorthogonalization (polfed:1022-1099)."""
    Qhist, Ablocks, Bblocks = [], [], []
    n = Q1.shape[0]
    Q = Q1.copy()
    Qprev = np.empty((n, 0))
    Bprev = np.empty((0, 0))
    for _ in range(mmax):
        Qhist.append(Q.copy())
        W = apply_poly_block(A, Q, coeffs, smin, smax, impl=impl)
        if Qprev.shape[1] > 0 and Bprev.shape[0] > 0 and Bprev.shape[1] > 0:
            W -= Qprev @ Bprev.T
        Aj = 0.5 * (Q.T @ W + W.T @ Q)
        Ablocks.append(Aj)
        W -= Q @ Aj
        for _ in range(reorth_passes):
            reorth_full(W, Qhist, Q, passes=1)
        Qnext, Bj = block_qr_factor(W, rtol)
        if Qnext.shape[1] == 0:
            break
        Bblocks.append(Bj)
        Qprev, Bprev, Q = Q, Bj, Qnext
    return Qhist, Ablocks, Bblocks


def extract_pairs(Qhist, Ablocks, Bblocks, A, *, nev, emin, emax, overextract=2, refine=True,
                  extra_keep=8, chunk=64, rtol=1e-12, impl="c"):
    """Reduced eigensolve, lift, interval filter, residual pruning (polfed:892-984)."""
    T = assemble_T(Ablocks, Bblocks)
    theta, U = np.linalg.eigh(T)
    m = min(theta.size, max(overextract * nev, nev + extra_keep))
    p = np.argsort(-theta, kind="stable")[:m]
    theta_sel = theta[p]
    Usel = U[:, p]
    n = Qhist[0].shape[0]
    lam_keep, res_keep, idx_keep = [], [], []
    for j0 in range(0, m, chunk):
        j1 = min(j0 + chunk, m)
        Xc = build_X(Qhist, Usel[:, j0:j1])
        lc, rc = rayleigh(A, Xc, impl=impl)
        for j in range(j1 - j0):
            if emin <= lc[j] <= emax:
                lam_keep.append(lc[j])
                res_keep.append(rc[j])
                idx_keep.append(j0 + j)
    empty = (np.empty(0), np.empty((n, 0)), np.empty(0), theta_sel)
    if not idx_keep:
        return empty
    lam_keep = np.array(lam_keep)
    res_keep = np.array(res_keep)
    idx_keep = np.array(idx_keep)
    npre = min(res_keep.size, nev + extra_keep)
    ps0 = np.argsort(res_keep, kind="stable")[:npre]
    lamc = lam_keep[ps0]
    resc = res_keep[ps0]
    idxc = idx_keep[ps0]
    Xc = build_X(Qhist, Usel[:, idxc])
    if refine:
        lamc, Xc, resc = refine_original_rr(A, Xc, rtol=1e-12, impl=impl)
        inside2 = (lamc >= emin) & (lamc <= emax)
        if not inside2.any():
            return empty
        lamc, resc, Xc = lamc[inside2], resc[inside2], Xc[:, inside2]
    nkeep = min(resc.size, nev + extra_keep)
    ps = np.argsort(resc, kind="stable")[:nkeep]
    lamf, Xf, rf = lamc[ps], Xc[:, ps], resc[ps]
    pe = np.argsort(lamf, kind="stable")
    return lamf[pe], Xf[:, pe], rf[pe], theta_sel


def polfed(A, nev: int, degree: int, *, s: int = 8, smin=None, smax=None, sigma: float = 0.0,
           emin: float = -math.inf, emax: float = math.inf, tol: float = 1e-10, threaded=True,
           overextract: int = 2, refine: bool = True, window_type: str = "step",
           jackson: bool = True, mmax: Optional[int] = None, rtol: float = 1e-12,
           reorth_passes: int = 1, extra_keep: int = 8, seed: int = 1,
           show_progress: bool = False, chunk: int = 64, impl: str = "c",
           Q0: Optional[np.ndarray] = None, info: Optional[dict] = None):
    """POLFED driver (polfed:1128-1158) with the reference's two-branch return rule."""
    n = A.shape[0]
    if smin is None or smax is None:
        raise ValueError("Matrix-free POLFED requires spectral bounds smin and smax")
    coeffs = build_coeffs(degree, smin, smax, sigma, emin, emax, window_type, jackson)
    if mmax is None:
        mmax = int(math.ceil(2.8 * nev / s))
    Q0 = splitmix_normal(seed, n, s) if Q0 is None else np.array(Q0, dtype=np.float64)
    Q1 = orth_block(Q0, rtol)
    Qhist, Ab, Bb = build_full_basis(A, Q1, coeffs, smin, smax, mmax, rtol, reorth_passes, impl)
    lam, X, res, _ = extract_pairs(Qhist, Ab, Bb, A, nev=nev, emin=emin, emax=emax,
                                   overextract=overextract, refine=refine,
                                   extra_keep=extra_keep, chunk=chunk, impl=impl)
    if info is not None:
        info["blocks"] = len(Qhist)
        info["basis_dim"] = sum(q.shape[1] for q in Qhist)
    if show_progress:
        _progress_line(len(Qhist), lam, res)
    if res.size and res.size >= nev:
        rs = np.sort(res)
        if rs[nev - 1] < tol:
            return lam[:nev], X[:, :nev], res[:nev]
    if res.size:
        p = np.argsort(res, kind="stable")[:min(nev, res.size)]
        return lam[p], X[:, p], res[p]
    return np.empty(0), np.empty((n, 0)), np.empty(0)


def _progress_line(m, lam, res):
    """polfed:991-1000."""
    if res.size == 0:
        print(f"m={m}  inside=0  maxres=Inf")
        return
    rs = np.sort(res)
    r90 = rs[min(max(int(round(0.9 * rs.size)), 1), rs.size) - 1]
    r95 = rs[min(max(int(round(0.95 * rs.size)), 1), rs.size) - 1]
    print(f"m={m}  inside={lam.size}  r90={r90}  r95={r95}  maxres={rs[-1]}")


# ======================================================================================
# Kernel polynomial method (no reference counterpart: the library's density-of-states
# extension).  Restated from the published method (Weisse, Wellein, Alvermann, Fehske,
# Rev. Mod. Phys. 78, 275 (2006), sections II.B-II.C) with the plain three-term
# recurrence -- not the doubling identities the GPU uses -- so the two checks differ in
# arithmetic.
# ======================================================================================
def kpm_moments(A, M: int, R: int, seed: int, smin: float, smax: float,
                per_vector: bool = False):
    """mu_k = (1/(n R)) sum_r z_r^T T_k(A_hat) z_r, k < M, Rademacher z_r."""
    from sparse_matrix_algorithms_b200.matrices import splitmix_rademacher

    n = A.shape[0]
    c = 0.5 * (smin + smax)
    d = 0.5 * (smax - smin)
    A = sp.csr_matrix(A)
    Z = splitmix_rademacher(seed, n, R)
    pv = np.empty((M, R))
    T0 = Z.copy()
    pv[0] = np.einsum("ij,ij->j", Z, T0)
    if M > 1:
        T1 = (A @ T0 - c * T0) / d
        pv[1] = np.einsum("ij,ij->j", Z, T1)
        for k in range(2, M):
            T2 = 2.0 * (A @ T1 - c * T1) / d - T0
            pv[k] = np.einsum("ij,ij->j", Z, T2)
            T0, T1 = T1, T2
    pv /= n
    mu = pv.mean(axis=1)
    return (mu, pv) if per_vector else mu


def kpm_count(mu, n: int, smin: float, smax: float, emin: float, emax: float,
              jackson: bool = True) -> float:
    """n times the integral over [emin, emax] of the damped Chebyshev density series."""
    M = len(mu)
    c = 0.5 * (smin + smax)
    d = 0.5 * (smax - smin)
    a = min(1.0, max(-1.0, (emin - c) / d))
    b = min(1.0, max(-1.0, (emax - c) / d))
    ta, tb = math.acos(a), math.acos(b)
    g = jackson_kernel(M - 1) if jackson else np.ones(M)
    k = np.arange(1, M)
    s = g[0] * mu[0] * (ta - tb) + np.sum(2.0 * g[1:] * np.asarray(mu[1:]) *
                                          (np.sin(k * ta) - np.sin(k * tb)) / k)
    return float(n * s / math.pi)


def divided_difference(c, t: float):
    """Chebyshev coefficients e of (p(s) - p(t)) / (s - t) for p = sum c_m T_m, and p(t).

    No counterpart in the reference (it is the FP32 polish of this library's MIXED POLFED).
    Computed here by numpy's Chebyshev-series long division of p - p(t) by (s - t), a route
    independent of the library's (the Clenshaw intermediates of p at t)."""
    from numpy.polynomial import chebyshev as C

    c = np.asarray(c, dtype=np.float64)
    pt = float(C.chebval(t, c))
    num = c.copy()
    num[0] -= pt
    q, _ = C.chebdiv(num, np.array([-t, 1.0]))
    e = np.zeros(len(c) - 1)
    e[:len(q)] = q
    return e, pt
