"""ctypes bindings of libsma (``include/sma.h``).

The library is loaded from the package directory (``libsma.so``, built in-tree by
``python -m sparse_matrix_algorithms_b200.build``).  There is no fallback: if the
library is missing or no CUDA device is present, calls fail with an exception.
"""
from __future__ import annotations

import ctypes
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libsma.so")

c_int64 = ctypes.c_int64
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
c_int = ctypes.c_int

# ------------------------------------------------------------------ status codes
SMA_OK = 0
SMA_ERR_ARG = 1
SMA_ERR_NONSYMMETRIC = 2
SMA_ERR_INTERVAL = 3
SMA_ERR_CUDA = 4
SMA_ERR_TIMEOUT = 5
SMA_ERR_NOCONV = 6
SMA_ERR_NOMEM = 7
SMA_ERR_BOUNDS = 8
SMA_ERR_WINDOW = 9
SMA_ERR_CALLBACK = 10
SMA_ERR_INTERNAL = 11

WINDOWS = {"step": 0, "delta": 1, "smooth": 2}
PRECISIONS = {"fp64": 0, "fp32": 1, "mixed": 2}


class SMAError(RuntimeError):
    """A libsma call failed; ``code`` is the status code."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class ArgumentError(SMAError, ValueError):
    """Julia's ArgumentError / error(...) on invalid arguments."""


class CudaError(SMAError):
    pass


# ------------------------------------------------------------------ structs
class ChebOpts(ctypes.Structure):
    _fields_ = [("smin", c_double), ("smax", c_double), ("has_bounds", c_int64),
                ("sigma", c_double), ("m0", c_int64), ("degree", c_int64),
                ("maxiter", c_int64), ("tol", c_double), ("res_gate", c_double),
                ("jackson", c_int64), ("debug", c_int64), ("two_hit", c_int64),
                ("seed", c_int64), ("window_type", c_int64), ("matrix_free", c_int64),
                ("precision", c_int64), ("lock", c_int64), ("reserved", c_int64 * 7)]


class PolfedOpts(ctypes.Structure):
    _fields_ = [("s", c_int64), ("smin", c_double), ("smax", c_double),
                ("has_bounds", c_int64), ("sigma", c_double), ("emin", c_double),
                ("emax", c_double), ("tol", c_double), ("threaded", c_int64),
                ("overextract", c_int64), ("refine", c_int64), ("window_type", c_int64),
                ("jackson", c_int64), ("mmax", c_int64), ("rtol", c_double),
                ("reorth_passes", c_int64), ("extra_keep", c_int64), ("seed", c_int64),
                ("show_progress", c_int64), ("chunk", c_int64), ("precision", c_int64),
                ("reserved", c_int64 * 8)]


class SliceOpts(ctypes.Structure):
    _fields_ = [("smin", c_double), ("smax", c_double), ("has_bounds", c_int64),
                ("maxiter", c_int64), ("tol", c_double), ("res_gate", c_double),
                ("jackson", c_int64), ("two_hit", c_int64), ("seed", c_int64),
                ("window_type", c_int64), ("precision", c_int64), ("graph", c_int64),
                ("debug", c_int64), ("reserved", c_int64 * 8)]


class Stats(ctypes.Structure):
    _fields_ = [("iterations", c_int64), ("basis_dim", c_int64), ("spmm_steps", c_int64),
                ("spmm_columns", c_int64), ("filter_ms", c_double), ("orth_ms", c_double),
                ("rr_ms", c_double), ("total_ms", c_double), ("filter_bytes", c_double),
                ("qr_fallbacks", c_int64), ("warnings", c_int64), ("kernel_launches", c_int64),
                ("fp32_filter_calls", c_int64), ("locked", c_int64),
                ("polish_iterations", c_int64), ("graph_replays", c_int64),
                ("polish_ms", c_double), ("polish_bytes", c_double),
                ("reserved", c_int64 * 1)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


MATBLOCK_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64,
                               c_void_p)

# (name, restype, argtypes) of every entry point declared in include/sma.h
SIGNATURES = [
    ("sma_abi_version", c_int, []),
    ("sma_last_error", ctypes.c_char_p, []),
    ("sma_kernel_launch_count", c_int64, []),
    ("sma_ctx_create", c_int, [c_int, ctypes.POINTER(c_void_p)]),
    ("sma_ctx_destroy", c_int, [c_void_p]),
    ("sma_ctx_synchronize", c_int, [c_void_p]),
    ("sma_ctx_stream", c_void_p, [c_void_p]),
    ("sma_op_create_csc", c_int, [c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_void_p,
                                  c_int64, c_int64, ctypes.POINTER(c_void_p)]),
    ("sma_op_create_csc_upper", c_int, [c_void_p, c_int64, c_int64, c_void_p, c_void_p,
                                        c_void_p, c_int64, c_int64, ctypes.POINTER(c_void_p)]),
    ("sma_op_create_lap1d", c_int, [c_void_p, c_int64, ctypes.POINTER(c_void_p)]),
    ("sma_op_create_anderson", c_int, [c_void_p, c_int64, c_void_p, c_double,
                                       ctypes.POINTER(c_void_p)]),
    ("sma_op_create_xxz", c_int, [c_void_p, c_int64, c_double, c_double, c_void_p,
                                  ctypes.POINTER(c_void_p)]),
    ("sma_op_create_matblock", c_int, [c_void_p, c_int64, MATBLOCK_FN, c_void_p,
                                       ctypes.POINTER(c_void_p)]),
    ("sma_op_destroy", c_int, [c_void_p]),
    ("sma_op_info", c_int, [c_void_p, ctypes.POINTER(c_int64), ctypes.POINTER(c_int64)]),
    ("sma_gershgorin_bounds", c_int, [c_void_p, ctypes.POINTER(c_double), ctypes.POINTER(c_double)]),
    ("sma_lanczos_bounds", c_int, [c_void_p, c_int64, c_int64, ctypes.POINTER(c_double),
                                   ctypes.POINTER(c_double)]),
    ("sma_jackson_kernel", c_int, [c_int64, c_void_p]),
    ("sma_cheb_delta_coeffs", c_int, [c_double, c_int64, c_int64, c_void_p]),
    ("sma_cheb_window_coeffs", c_int, [c_double, c_double, c_int64, c_int64, c_void_p]),
    ("sma_cheb_smooth_window_coeffs", c_int, [c_double, c_double, c_int64, c_int64, c_int64,
                                              c_double, c_void_p]),
    ("sma_build_coeffs", c_int, [c_int64, c_double, c_double, c_double, c_double, c_double,
                                 c_int64, c_int64, c_void_p]),
    ("sma_apply_poly_block_dev", c_int, [c_void_p, c_void_p, c_int64, c_double, c_double,
                                         c_void_p, c_int64, c_void_p, c_int64, c_int64, c_int64]),
    ("sma_apply_poly_block", c_int, [c_void_p, c_void_p, c_int64, c_double, c_double, c_void_p,
                                     c_void_p, c_int64, c_int64]),
    ("sma_spmm_dev", c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_int64]),
    ("sma_apply_poly_block_percol_dev", c_int, [c_void_p, c_void_p, c_int64, c_double, c_double,
                                                c_void_p, c_void_p, c_int64, c_int64]),
    ("sma_dense_gram_dev", c_int, [c_void_p, c_int64, c_int64, c_int64, c_void_p, c_int64,
                                   c_void_p, c_int64, c_void_p, c_int64, c_double, c_double]),
    ("sma_dense_update_dev", c_int, [c_void_p, c_int64, c_int64, c_int64, c_void_p, c_int64,
                                     c_void_p, c_int64, c_int64, c_void_p, c_int64, c_double,
                                     c_double]),
    ("sma_divided_difference", c_int, [c_void_p, c_int64, c_double, c_void_p, c_void_p]),
    ("sma_apply_poly_block_noalloc", c_int, [c_void_p, c_void_p, c_int64, c_double, c_double,
                                             c_void_p, c_int64, c_void_p, c_int64, c_int64]),
    ("sma_kpm_moments", c_int, [c_void_p, c_int64, c_int64, c_int64, c_double, c_double,
                                c_void_p, c_void_p]),
    ("sma_kpm_count", c_int, [c_void_p, c_int64, c_int64, c_double, c_double, c_double,
                              c_double, c_int64, ctypes.POINTER(c_double)]),
    ("sma_cheb_opts_default", None, [ctypes.POINTER(ChebOpts)]),
    ("sma_polfed_opts_default", None, [ctypes.POINTER(PolfedOpts)]),
    ("sma_cheb_solve", c_int, [c_void_p, c_double, c_double, ctypes.POINTER(ChebOpts),
                               ctypes.POINTER(c_void_p)]),
    ("sma_polfed_solve", c_int, [c_void_p, c_int64, c_int64, ctypes.POINTER(PolfedOpts),
                                 ctypes.POINTER(c_void_p)]),
    ("sma_polfed_batch_solve", c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_void_p)]),
    ("sma_slice_opts_default", None, [ctypes.POINTER(SliceOpts)]),
    ("sma_slice_solve", c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                ctypes.POINTER(SliceOpts), ctypes.POINTER(c_void_p)]),
    ("sma_mlp_create", c_int, [c_void_p, c_int64, c_int64, c_int64, c_int64,
                               ctypes.POINTER(c_void_p)]),
    ("sma_mlp_destroy", c_int, [c_void_p]),
    ("sma_mlp_num_params", c_int, [c_void_p, ctypes.POINTER(c_int64)]),
    ("sma_mlp_get_params", c_int, [c_void_p, c_void_p]),
    ("sma_mlp_set_params", c_int, [c_void_p, c_void_p]),
    ("sma_mlp_forward", c_int, [c_void_p, c_void_p, c_int64, c_void_p]),
    ("sma_mlp_grad", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                             ctypes.POINTER(ctypes.c_float), c_void_p]),
    ("sma_mlp_train", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int64,
                              c_double, c_int64, c_int64, c_double, c_void_p]),
    ("sma_selftest_barrier_timeout", c_int, [c_void_p, ctypes.POINTER(c_int64)]),
    ("sma_result_count", c_int, [c_void_p, ctypes.POINTER(c_int64), ctypes.POINTER(c_int64)]),
    ("sma_result_copy", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sma_result_stats", c_int, [c_void_p, ctypes.POINTER(Stats)]),
    ("sma_result_windows", c_int, [c_void_p, c_void_p]),
    ("sma_result_window_info", c_int, [c_void_p, c_int64, c_void_p, c_void_p]),
    ("sma_result_free", c_int, [c_void_p]),
]

_lib = None
_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Load libsma.so (once).  Raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with "
                    "`python -m sparse_matrix_algorithms_b200.build` (nvcc, sm_100a)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, restype, argtypes in SIGNATURES:
                fn = getattr(lib, name)
                fn.restype = restype
                fn.argtypes = argtypes
            _lib = lib
    return _lib


_ERRORS = {SMA_ERR_ARG: ArgumentError, SMA_ERR_NONSYMMETRIC: ArgumentError,
           SMA_ERR_INTERVAL: ArgumentError, SMA_ERR_BOUNDS: ArgumentError,
           SMA_ERR_WINDOW: ArgumentError, SMA_ERR_CUDA: CudaError}


def check(rc: int) -> None:
    """Raise the exception matching a libsma status code."""
    if rc == SMA_OK:
        return
    msg = (load().sma_last_error() or b"").decode(errors="replace")
    if rc == SMA_ERR_NOMEM:
        raise MemoryError(msg)
    raise _ERRORS.get(rc, SMAError)(rc, msg)
