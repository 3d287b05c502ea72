"""Python mirror of the reference's public API, running on the CUDA library.

Names, keyword arguments, defaults, return values and error behaviour follow
``chebyshev_subspace_iteration.jl`` and ``polfed.jl``:

* :func:`chebyshev_poly_real_symm_sparse` -- both overloads
  (sparse matrix, ``chebyshev_subspace_iteration.jl:667``; matrix-free
  ``(matvec, n, emin, emax; matblock=...)``, ``chebyshev_subspace_iteration.jl:771``);
* :func:`polfed` -- ``polfed(A::MatrixFreeRealSymOp, nev, degree; ...)`` (``polfed.jl:1128``)
  and ``polfed(matvec, n, nev, degree; matblock=...)`` (``polfed.jl:1183``);
* :class:`MatrixFreeRealSymOp` (``polfed.jl:148-165``), :func:`gershgorin_bounds`,
  :func:`jackson_kernel`, :func:`cheb_delta_coeffs`, :func:`cheb_window_coeffs`,
  :func:`cheb_smooth_window_coeffs`, :func:`build_coeffs` (``_build_coeffs``) and
  :func:`apply_poly_block`.

Every numerical step runs in ``libsma.so`` on the GPU.  Matrix-free operators must be
device operators (a built-in stencil, a device CSR matrix, or a callback that enqueues
GPU work); a host ``matvec!`` closure is rejected rather than run on the CPU.
"""
from __future__ import annotations

import ctypes
import math
from typing import Callable, Optional

import numpy as np
import scipy.sparse as sp

from . import _lib as L

__all__ = [
    "Context", "context", "SparseOperator", "Lap1dOperator", "AndersonOperator", "XXZOperator",
    "DeviceMatblock",
    "MatrixFreeRealSymOp", "chebyshev_poly_real_symm_sparse", "polfed", "gershgorin_bounds",
    "jackson_kernel", "cheb_delta_coeffs", "cheb_window_coeffs", "cheb_smooth_window_coeffs",
    "build_coeffs", "apply_poly_block", "lanczos_bounds", "polfed_windows", "ArgumentError",
    "SMAError",
]

ArgumentError = L.ArgumentError
SMAError = L.SMAError
_LIB = L  # for methods whose arguments are named L (lattice / chain length)


# ====================================================================== context
class Context:
    """A CUDA stream plus cuBLAS/cuSOLVER handles on one device (``sma_ctx``)."""

    def __init__(self, device: int = 0):
        self._lib = L.load()
        h = ctypes.c_void_p()
        L.check(self._lib.sma_ctx_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.device = device

    @property
    def stream(self) -> int:
        return self._lib.sma_ctx_stream(self.handle) or 0

    def synchronize(self) -> None:
        L.check(self._lib.sma_ctx_synchronize(self.handle))

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.sma_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_CONTEXTS: dict = {}


def context(device: int = 0) -> Context:
    """The process-wide default context of ``device``."""
    ctx = _CONTEXTS.get(device)
    if ctx is None:
        ctx = _CONTEXTS[device] = Context(device)
    return ctx


# ====================================================================== operators
class _DeviceOp:
    handle: ctypes.c_void_p
    n: int

    @property
    def shape(self):
        return (self.n, self.n)

    def close(self) -> None:
        if getattr(self, "handle", None):
            L.load().sma_op_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SparseOperator(_DeviceOp):
    """Device copy of a sparse symmetric matrix (its CSC arrays, which for a symmetric
    matrix are also its CSR arrays).  ``check_symmetric`` verifies A == A^T exactly.
    ``storage="upper"`` keeps only the upper triangle on the device (symmetric half
    storage, ``sma_op_create_csc_upper``): about half the memory, products equal to full
    storage up to rounding."""

    def __init__(self, A, ctx: Optional[Context] = None, check_symmetric: bool = False,
                 storage: str = "full"):
        if storage not in ("full", "upper"):
            raise ArgumentError(L.SMA_ERR_ARG, "storage must be 'full' or 'upper'")
        self.storage = storage
        self.ctx = ctx or context()
        C = sp.csc_matrix(A, dtype=np.float64)
        if C.shape[0] != C.shape[1]:
            raise ArgumentError(L.SMA_ERR_ARG, "A must be square")
        C.sum_duplicates()
        C.sort_indices()
        self.n = C.shape[0]
        self.nnz = C.nnz
        colptr = np.ascontiguousarray(C.indptr, dtype=np.int64)
        rowval = np.ascontiguousarray(C.indices, dtype=np.int64)
        nzval = np.ascontiguousarray(C.data, dtype=np.float64)
        h = ctypes.c_void_p()
        create = (L.load().sma_op_create_csc if storage == "full"
                  else L.load().sma_op_create_csc_upper)
        L.check(create(self.ctx.handle, self.n, self.nnz, colptr.ctypes.data, rowval.ctypes.data,
                       nzval.ctypes.data, 0, int(bool(check_symmetric)), ctypes.byref(h)))
        self.handle = h
        if storage == "upper":
            stored = ctypes.c_int64()
            L.check(L.load().sma_op_info(self.handle, None, ctypes.byref(stored)))
            self.nnz_stored = stored.value
        else:
            self.nnz_stored = self.nnz

    def gershgorin_bounds(self):
        lo, hi = ctypes.c_double(), ctypes.c_double()
        L.check(L.load().sma_gershgorin_bounds(self.handle, ctypes.byref(lo), ctypes.byref(hi)))
        return lo.value, hi.value


class Lap1dOperator(_DeviceOp):
    """tridiag(-1, 2, -1) as a device stencil: the GPU form of the reference's
    ``lap1d_matblock!`` (``polfed.jl:1209-1219``)."""

    def __init__(self, n: int, ctx: Optional[Context] = None):
        self.ctx = ctx or context()
        self.n = int(n)
        h = ctypes.c_void_p()
        L.check(L.load().sma_op_create_lap1d(self.ctx.handle, self.n, ctypes.byref(h)))
        self.handle = h


class AndersonOperator(_DeviceOp):
    """The 3D Anderson model of :func:`matrices.anderson3d` (same L, W, seed) as a device
    stencil: no stored matrix, products bit-identical to the CSR matrix's."""

    def __init__(self, L: int, W: float, seed: int, t: float = -1.0,
                 ctx: Optional[Context] = None):
        from .matrices import splitmix_uniform

        self.ctx = ctx or context()
        self.n = int(L) ** 3
        eps = np.ascontiguousarray(W * (splitmix_uniform(seed, self.n) - 0.5))
        h = ctypes.c_void_p()
        _LIB.check(_LIB.load().sma_op_create_anderson(self.ctx.handle, int(L), eps.ctypes.data,
                                                      float(t), ctypes.byref(h)))
        self.handle = h


class XXZOperator(_DeviceOp):
    """The random-field XXZ chain of :func:`matrices.xxz_sz0` (same L, h, seed, J, Delta)
    in the Sz = 0 sector as a device stencil (no stored matrix)."""

    def __init__(self, L: int, h: float, seed: int, J: float = 1.0, Delta: float = 1.0,
                 ctx: Optional[Context] = None):
        from .matrices import splitmix_uniform
        from math import comb

        self.ctx = ctx or context()
        self.n = comb(int(L), int(L) // 2)
        field = np.ascontiguousarray(h * (2.0 * splitmix_uniform(seed, L) - 1.0))
        hd = ctypes.c_void_p()
        _LIB.check(_LIB.load().sma_op_create_xxz(self.ctx.handle, int(L), float(J), float(Delta),
                                                 field.ctypes.data, ctypes.byref(hd)))
        self.handle = hd


class DeviceMatblock(_DeviceOp):
    """Matrix-free operator from a device block callback.

    ``fn(X_ptr, Y_ptr, n, b, ld, stream)`` must enqueue ``Y = A X`` for the row-major
    n x b FP64 device blocks at ``X_ptr``/``Y_ptr`` (leading dimension ``ld``) on the
    CUDA stream ``stream`` and return 0 (or None).
    """

    def __init__(self, n: int, fn: Callable, ctx: Optional[Context] = None):
        self.ctx = ctx or context()
        self.n = int(n)
        self._fn = fn

        def tramp(_user, x, y, nn, b, ld, stream):
            try:
                rc = fn(x or 0, y or 0, int(nn), int(b), int(ld), stream or 0)
                return int(rc or 0)
            except Exception:  # an exception must not cross into C
                return 1

        self._cb = L.MATBLOCK_FN(tramp)
        h = ctypes.c_void_p()
        L.check(L.load().sma_op_create_matblock(self.ctx.handle, self.n, self._cb, None,
                                                ctypes.byref(h)))
        self.handle = h


class MatrixFreeRealSymOp:
    """``MatrixFreeRealSymOp(n, matvec!, matblock!)`` (``polfed.jl:148-165``).

    The block action must be a device operator: :class:`Lap1dOperator`,
    :class:`SparseOperator`, :class:`DeviceMatblock`, or a callable carrying
    ``device_block = True`` (wrapped as :class:`DeviceMatblock`).  ``matvec`` is kept
    for signature compatibility; without a device block action the constructor
    raises, since host closures are never executed.
    """

    def __init__(self, n: int, matvec=None, matblock=None):
        self.n = int(n)
        self.matvec = matvec
        self.matblock = matblock
        self.device_op = _as_device_op(self.n, matblock if matblock is not None else matvec)

    @property
    def shape(self):
        return (self.n, self.n)


def _as_device_op(n: int, f) -> _DeviceOp:
    if isinstance(f, _DeviceOp):
        if f.n != n:
            raise ArgumentError(L.SMA_ERR_ARG, f"operator dimension {f.n} != n = {n}")
        return f
    if callable(f) and getattr(f, "device_block", False):
        return DeviceMatblock(n, f)
    raise ArgumentError(
        L.SMA_ERR_ARG,
        "matrix-free operators must act on device blocks (Lap1dOperator, SparseOperator, "
        "DeviceMatblock or a callable with device_block=True); host matvec!/matblock! "
        "closures are not run")


def _resolve_sparse(A):
    if isinstance(A, SparseOperator):
        return A
    if sp.issparse(A):
        return SparseOperator(A)
    raise TypeError(f"expected a scipy sparse matrix or SparseOperator, got {type(A).__name__}")


# ====================================================================== coefficients
def _coeff_call(fn, K, *args):
    out = np.empty(K + 1, dtype=np.float64)
    L.check(fn(*args, out.ctypes.data))
    return out


def jackson_kernel(K: int) -> np.ndarray:
    """Jackson damping g_0..g_K (``chebyshev_subspace_iteration.jl:376``)."""
    n = max(K, 0)
    out = np.empty(n + 1)
    L.check(L.load().sma_jackson_kernel(int(K), out.ctypes.data))
    return out


def cheb_delta_coeffs(sigma_hat: float, K: int, jackson: bool = True) -> np.ndarray:
    return _coeff_call(L.load().sma_cheb_delta_coeffs, K, float(sigma_hat), int(K), int(jackson))


def cheb_window_coeffs(a: float, b: float, K: int, jackson: bool = True) -> np.ndarray:
    return _coeff_call(L.load().sma_cheb_window_coeffs, K, float(a), float(b), int(K), int(jackson))


def cheb_smooth_window_coeffs(a: float, b: float, K: int, jackson: bool = True,
                              nsamp: int = 4096, delta: float = 0.02) -> np.ndarray:
    return _coeff_call(L.load().sma_cheb_smooth_window_coeffs, K, float(a), float(b), int(K),
                       int(jackson), int(nsamp), float(delta))


def build_coeffs(degree: int, smin: float, smax: float, sigma: float, emin: float, emax: float,
                 window_type: str = "step", jackson: bool = True) -> np.ndarray:
    """``_build_coeffs`` (``polfed.jl:404-414``)."""
    return _coeff_call(L.load().sma_build_coeffs, degree, int(degree), float(smin), float(smax),
                       float(sigma), float(emin), float(emax), _window(window_type), int(jackson))


def _window(window_type) -> int:
    key = str(window_type).lstrip(":")
    if key not in L.WINDOWS:
        raise ArgumentError(L.SMA_ERR_WINDOW, f"Unknown window type: {window_type}")
    return L.WINDOWS[key]


def gershgorin_bounds(A):
    """Gershgorin bounds of an explicit sparse matrix (``chebyshev_subspace_iteration.jl:351``)."""
    if isinstance(A, MatrixFreeRealSymOp):
        raise ArgumentError(L.SMA_ERR_ARG, "gershgorin_bounds needs an explicit sparse matrix")
    return _resolve_sparse(A).gershgorin_bounds()


def lanczos_bounds(A, steps: int = 60, seed: int = 7):
    """Spectral bounds from ``steps`` GPU Lanczos steps (an extension of the reference,
    which has only Gershgorin bounds); clipped to the Gershgorin interval for matrices."""
    op = _op_of(A)
    lo, hi = ctypes.c_double(), ctypes.c_double()
    L.check(L.load().sma_lanczos_bounds(op.handle, int(steps), int(seed), ctypes.byref(lo),
                                        ctypes.byref(hi)))
    return lo.value, hi.value


# ====================================================================== the filter
def apply_poly_block(A, Q: np.ndarray, coeffs, smin: float, smax: float,
                     precision: str = "fp64") -> np.ndarray:
    """Y = p(A_hat) Q (``apply_poly_block!``, ``chebyshev_subspace_iteration.jl:554``) on the
    GPU; ``Q`` is an n x b host array, the result an n x b Fortran-ordered array."""
    op = _op_of(A)
    Qf = np.asfortranarray(Q, dtype=np.float64)
    if Qf.ndim != 2 or Qf.shape[0] != op.n:
        raise ArgumentError(L.SMA_ERR_ARG, "Q must be n x b")
    Y = np.empty_like(Qf, order="F")
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    L.check(L.load().sma_apply_poly_block(op.handle, c.ctypes.data, len(c) - 1, float(smin),
                                          float(smax), Qf.ctypes.data, Y.ctypes.data,
                                          Qf.shape[1], L.PRECISIONS[precision]))
    return Y


def _op_of(A) -> _DeviceOp:
    if isinstance(A, MatrixFreeRealSymOp):
        return A.device_op
    if isinstance(A, _DeviceOp):
        return A
    return _resolve_sparse(A)


# ====================================================================== results
def _take_result(hres: ctypes.c_void_p, stats: Optional[dict], vectors: bool = True):
    """(lam, X, res) of a result handle, which is freed.  ``vectors=False`` leaves the
    eigenvectors on the device (X is None): no n x k download."""
    lib = L.load()
    try:
        k, n = ctypes.c_int64(), ctypes.c_int64()
        L.check(lib.sma_result_count(hres, ctypes.byref(k), ctypes.byref(n)))
        lam = np.empty(k.value)
        res = np.empty(k.value)
        X = np.empty((n.value, k.value), order="F") if vectors else None
        L.check(lib.sma_result_copy(hres, lam.ctypes.data,
                                    X.ctypes.data if X is not None and X.size else None,
                                    res.ctypes.data))
        if stats is not None:
            st = L.Stats()
            L.check(lib.sma_result_stats(hres, ctypes.byref(st)))
            stats.update(st.as_dict())
    finally:
        lib.sma_result_free(hres)
    return lam, X, res


# ====================================================================== Chebyshev
def chebyshev_poly_real_symm_sparse(A, *args, smin=None, smax=None, sigma: float = 0.0,
                                    m0: int = 200, degree: int = 80, maxiter: int = 8,
                                    tol: float = 1e-10, res_gate: float = 1e-6,
                                    jackson: bool = True, debug: bool = False,
                                    two_hit: bool = True, seed: int = 1,
                                    window_type="step", matblock=None, precision: str = "fp64",
                                    lock: bool = False, stats: Optional[dict] = None, **kw):
    """Chebyshev-filtered subspace iteration.

    ``chebyshev_poly_real_symm_sparse(A, emin, emax; ...)`` with a sparse matrix (or
    :class:`SparseOperator`): the sparse overload, which always runs ``maxiter``
    iterations (``chebyshev_subspace_iteration.jl:667-757``).

    ``chebyshev_poly_real_symm_sparse(matvec, n, emin, emax; matblock=...)`` or with a
    :class:`MatrixFreeRealSymOp` first: the matrix-free overload, which stops on the
    ``two_hit`` rule (``chebyshev_subspace_iteration.jl:771-848``).

    Returns ``(lam, X, res)`` sorted by lambda, with absolute residuals.  ``sigma`` may
    also be passed as ``σ``.  Extensions: ``precision="fp32"`` runs the filter in FP32,
    ``"mixed"`` in FP32 until the residuals stop improving and in FP64 after that;
    ``lock=True`` locks converged pairs (stopping on the matrix-free ``two_hit`` rule).
    """
    if "σ" in kw:
        sigma = kw.pop("σ")
    if kw:
        raise TypeError(f"unexpected keyword arguments {sorted(kw)}")
    if isinstance(A, MatrixFreeRealSymOp):
        op, (emin, emax), mf = A.device_op, args, True
    elif isinstance(A, _DeviceOp) and not isinstance(A, SparseOperator):  # device stencil
        op, (emin, emax), mf = A, args, True
    elif sp.issparse(A) or isinstance(A, SparseOperator):
        if matblock is not None:
            raise TypeError("matblock is a keyword of the matrix-free overload")
        op, (emin, emax), mf = _resolve_sparse(A), args, False
    else:  # (matvec!, n, emin, emax)
        n, emin, emax = args
        op, mf = MatrixFreeRealSymOp(n, A, matblock).device_op, True
    o = L.ChebOpts()
    L.load().sma_cheb_opts_default(ctypes.byref(o))
    if smin is not None and smax is not None:
        o.smin, o.smax, o.has_bounds = float(smin), float(smax), 1
    o.sigma = float(sigma)
    o.m0, o.degree, o.maxiter = int(m0), int(degree), int(maxiter)
    o.tol, o.res_gate = float(tol), float(res_gate)
    o.jackson, o.debug, o.two_hit, o.seed = int(jackson), int(debug), int(two_hit), int(seed)
    o.window_type = _window(window_type)
    o.matrix_free = int(mf)
    o.precision = L.PRECISIONS[precision]
    o.lock = int(bool(lock))
    h = ctypes.c_void_p()
    L.check(L.load().sma_cheb_solve(op.handle, float(emin), float(emax), ctypes.byref(o),
                                    ctypes.byref(h)))
    return _take_result(h, stats)


# ====================================================================== POLFED
def polfed(A, *args, s: int = 8, smin=None, smax=None, sigma: float = 0.0,
           emin: float = -math.inf, emax: float = math.inf, tol: float = 1e-10,
           threaded: bool = True, overextract: int = 2, refine: bool = True,
           window_type="step", jackson: bool = True, mmax: Optional[int] = None,
           rtol: float = 1e-12, reorth_passes: int = 1, extra_keep: int = 8, seed: int = 1,
           show_progress: bool = False, chunk: int = 64, precision: str = "fp64",
           stats: Optional[dict] = None, vectors: bool = True, **kw):
    """POLFED: block Lanczos on the Chebyshev-filtered operator (``polfed.jl:1128``).

    ``polfed(A, nev, degree; ...)`` with a :class:`MatrixFreeRealSymOp` (or, as an
    extension the reference lacks, a sparse matrix / :class:`SparseOperator`), or
    ``polfed(matvec, n, nev, degree; matblock=...)`` (``polfed.jl:1183``; ``matblock!``
    may be spelled ``matblock``).  ``smin``/``smax`` are required.  The return order
    follows ``polfed.jl:1148-1157``: by eigenvalue when the nev-th smallest residual is
    below ``tol``, else the nev best by residual.  ``vectors=False`` returns X as None
    (the eigenvectors are not copied to the host).
    """
    matblock = kw.pop("matblock!", kw.pop("matblock", None))
    if kw:
        raise TypeError(f"unexpected keyword arguments {sorted(kw)}")
    if isinstance(A, MatrixFreeRealSymOp):
        op, (nev, degree) = A.device_op, args
    elif sp.issparse(A) or isinstance(A, _DeviceOp):
        op, (nev, degree) = _op_of(A), args
    else:
        n, nev, degree = args
        op = MatrixFreeRealSymOp(n, A, matblock).device_op
    o = L.PolfedOpts()
    L.load().sma_polfed_opts_default(ctypes.byref(o))
    o.s = int(s)
    if smin is not None and smax is not None:
        o.smin, o.smax, o.has_bounds = float(smin), float(smax), 1
    o.sigma, o.emin, o.emax, o.tol = float(sigma), float(emin), float(emax), float(tol)
    o.threaded, o.overextract, o.refine = int(threaded), int(overextract), int(refine)
    o.window_type, o.jackson = _window(window_type), int(jackson)
    o.mmax = 0 if mmax is None else int(mmax)
    o.rtol, o.reorth_passes, o.extra_keep = float(rtol), int(reorth_passes), int(extra_keep)
    o.seed, o.show_progress, o.chunk = int(seed), int(show_progress), int(chunk)
    o.precision = L.PRECISIONS[precision]
    h = ctypes.c_void_p()
    L.check(L.load().sma_polfed_solve(op.handle, int(nev), int(degree), ctypes.byref(o),
                                      ctypes.byref(h)))
    return _take_result(h, stats, vectors)


# ====================================================================== batched POLFED
def polfed_windows(A, windows, nevs, degrees, mmaxs, *, s: int = 8, smin=None, smax=None,
                   tol: float = 1e-10, overextract: int = 2, refine: bool = True,
                   window_type="step", jackson: bool = True, rtol: float = 1e-12,
                   reorth_passes: int = 1, extra_keep: int = 8, seed: int = 1,
                   show_progress: bool = False, precision: str = "fp64",
                   stats: Optional[dict] = None, vectors: bool = True):
    """Batched POLFED (an extension; the reference runs ``polfed`` on one window per call):
    window ``w`` = ``windows[w]`` is a POLFED solve with ``nevs[w]``, ``degrees[w]`` and
    ``mmaxs[w]`` (its filter centred on the window, seed ``seed + w``), and every block step
    filters all windows' blocks in ONE segmented recurrence.  Returns
    ``(lam, X, res, win)``: per window its pairs in polfed's return order, windows in
    order, ``win[j]`` the window of pair ``j``.  ``stats`` also receives
    ``window_blocks`` and ``window_by_lambda`` (the return rule's branch) per window."""
    op = A if isinstance(A, _DeviceOp) else _resolve_sparse(A)
    w = np.asarray(windows, dtype=np.float64).reshape(-1, 2)
    emin = np.ascontiguousarray(w[:, 0])
    emax = np.ascontiguousarray(w[:, 1])
    nev = np.ascontiguousarray(nevs, dtype=np.int64)
    deg = np.ascontiguousarray(degrees, dtype=np.int64)
    mm = np.ascontiguousarray(mmaxs, dtype=np.int64)
    if not (nev.size == deg.size == mm.size == emin.size):
        raise ArgumentError(L.SMA_ERR_ARG, "windows, nevs, degrees and mmaxs differ in length")
    if smin is None or smax is None:
        raise ArgumentError(L.SMA_ERR_BOUNDS, "Matrix-free POLFED requires spectral bounds smin and smax")
    o = L.PolfedOpts()
    lib = L.load()
    lib.sma_polfed_opts_default(ctypes.byref(o))
    o.s, o.smin, o.smax, o.has_bounds = int(s), float(smin), float(smax), 1
    o.tol, o.overextract, o.refine = float(tol), int(overextract), int(refine)
    o.window_type, o.jackson = _window(window_type), int(jackson)
    o.rtol, o.reorth_passes, o.extra_keep = float(rtol), int(reorth_passes), int(extra_keep)
    o.seed, o.show_progress = int(seed), int(show_progress)
    o.precision = L.PRECISIONS[precision]
    h = ctypes.c_void_p()
    L.check(lib.sma_polfed_batch_solve(op.handle, int(emin.size), emin.ctypes.data,
                                       emax.ctypes.data, nev.ctypes.data, deg.ctypes.data,
                                       mm.ctypes.data, ctypes.byref(o), ctypes.byref(h)))
    k = ctypes.c_int64()
    L.check(lib.sma_result_count(h, ctypes.byref(k), None))
    win = np.zeros(k.value, dtype=np.int64)
    if k.value:
        L.check(lib.sma_result_windows(h, win.ctypes.data))
    if stats is not None:
        its = np.zeros(emin.size, dtype=np.int64)
        conv = np.zeros(emin.size, dtype=np.int64)
        L.check(lib.sma_result_window_info(h, int(emin.size), its.ctypes.data, conv.ctypes.data))
        stats["window_blocks"] = its
        stats["window_by_lambda"] = conv.astype(bool)
    lam, X, res = _take_result(h, stats, vectors)
    return lam, X, res, win


# ====================================================================== batched slicing
def slice_spectrum(A, windows, degrees, m0s, *, smin=None, smax=None, maxiter: int = 8,
                   tol: float = 1e-10, res_gate: float = 1e-6, jackson: bool = True,
                   two_hit: bool = True, seed: int = 1, window_type="step",
                   precision: str = "fp64", graph: bool = True, debug: bool = False,
                   stats: Optional[dict] = None):
    """Batched spectrum slicing (an extension; the reference solves one window per call).

    ``windows`` is a sequence of ``(emin, emax)``; window ``w`` runs Chebyshev subspace
    iteration with degree ``degrees[w]`` and width ``m0s[w]`` (rounded up to a multiple
    of 8), seed ``seed + w`` and the matrix-free overload's termination rule, and every
    iteration filters all unconverged windows in ONE batched recurrence (graph-captured
    when ``graph``).  Returns ``(lam, X, res, win)``: per window its pairs by eigenvalue,
    windows in order, ``win[j]`` the window of pair ``j``.
    """
    op = A if isinstance(A, _DeviceOp) else _resolve_sparse(A)
    w = np.asarray(windows, dtype=np.float64).reshape(-1, 2)
    emin = np.ascontiguousarray(w[:, 0])
    emax = np.ascontiguousarray(w[:, 1])
    deg = np.ascontiguousarray(degrees, dtype=np.int64)
    m0 = np.ascontiguousarray(m0s, dtype=np.int64)
    if not (deg.size == m0.size == emin.size):
        raise ArgumentError(L.SMA_ERR_ARG, "windows, degrees and m0s differ in length")
    o = L.SliceOpts()
    lib = L.load()
    lib.sma_slice_opts_default(ctypes.byref(o))
    if smin is not None and smax is not None:
        o.smin, o.smax, o.has_bounds = float(smin), float(smax), 1
    o.maxiter, o.tol, o.res_gate = int(maxiter), float(tol), float(res_gate)
    o.jackson, o.two_hit, o.seed = int(jackson), int(two_hit), int(seed)
    o.window_type, o.precision = _window(window_type), L.PRECISIONS[precision]
    o.graph, o.debug = int(graph), int(debug)
    h = ctypes.c_void_p()
    L.check(lib.sma_slice_solve(op.handle, int(emin.size), emin.ctypes.data, emax.ctypes.data,
                                deg.ctypes.data, m0.ctypes.data, ctypes.byref(o),
                                ctypes.byref(h)))
    k = ctypes.c_int64()
    L.check(lib.sma_result_count(h, ctypes.byref(k), None))
    win = np.zeros(k.value, dtype=np.int64)
    if k.value:
        L.check(lib.sma_result_windows(h, win.ctypes.data))
    if stats is not None:
        its = np.zeros(emin.size, dtype=np.int64)
        conv = np.zeros(emin.size, dtype=np.int64)
        L.check(lib.sma_result_window_info(h, int(emin.size), its.ctypes.data, conv.ctypes.data))
        stats["window_iterations"] = its
        stats["window_converged"] = conv.astype(bool)
    lam, X, res = _take_result(h, stats)
    return lam, X, res, win


# ====================================================================== KPM density of states
def kpm_moments(A, M: int = 256, R: int = 16, *, smin=None, smax=None, seed: int = 11,
                per_vector: bool = False):
    """Stochastic Chebyshev moments ``mu[0..M-1]`` of the spectral density of ``A`` on the
    GPU (an extension: the reference has no density-of-states estimate).  ``R``
    Rademacher vectors; ``[smin, smax]`` defaults to the Gershgorin bounds.  With
    ``per_vector`` also returns the ``M x R`` per-vector moments."""
    op = _op_of(A)
    if smin is None or smax is None:
        if not hasattr(op, "gershgorin_bounds"):
            raise ArgumentError(L.SMA_ERR_ARG, "pass smin and smax for a matrix-free operator")
        smin, smax = op.gershgorin_bounds()
    mu = np.empty(int(M))
    pv = np.empty((int(M), int(R))) if per_vector else None
    L.check(L.load().sma_kpm_moments(op.handle, int(M), int(R), int(seed), float(smin),
                                     float(smax), mu.ctypes.data,
                                     pv.ctypes.data if pv is not None else None))
    return (mu, pv) if per_vector else mu


def kpm_count(mu, n: int, smin: float, smax: float, emin: float, emax: float,
              jackson: bool = True) -> float:
    """Eigenvalue count in ``[emin, emax]`` predicted by KPM moments of an n x n matrix."""
    m = np.ascontiguousarray(mu, dtype=np.float64)
    out = ctypes.c_double()
    L.check(L.load().sma_kpm_count(m.ctypes.data, int(m.size), int(n), float(smin),
                                   float(smax), float(emin), float(emax), int(jackson),
                                   ctypes.byref(out)))
    return out.value
