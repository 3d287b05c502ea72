"""CPU-side checks of the C ABI: the library loads, exports every entry point that
include/sma.h declares, its host-only functions agree with the oracle, and compute
calls fail loudly (never fall back) when no GPU is usable."""
import ctypes
import os
import re

import numpy as np
import pytest

import sma_oracle as O
from conftest import ROOT


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "sma.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(sma_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_declares_the_solver_surface():
    names = _declared_functions()
    for required in ["sma_cheb_solve", "sma_polfed_solve", "sma_apply_poly_block",
                     "sma_apply_poly_block_dev", "sma_op_create_csc", "sma_result_copy",
                     "sma_last_error"]:
        assert required in names


def test_library_exports_every_declared_symbol(lib_built):
    lib = ctypes.CDLL(lib_built)
    missing = [n for n in _declared_functions() if not hasattr(lib, n)]
    assert missing == []


def test_python_bindings_cover_the_header(lib_built):
    from sparse_matrix_algorithms_b200 import _lib as L

    bound = {name for name, _, _ in L.SIGNATURES}
    assert bound == set(_declared_functions())
    L.load()


def _header_struct_members(name):
    """Member names (reserved arrays expanded) of `typedef struct name {...}` in sma.h."""
    src = open(os.path.join(ROOT, "include", "sma.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, flags=re.S).group(1)
    members = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        typ, rest = decl.split(None, 1)
        assert typ in ("int64_t", "double"), decl
        for m in rest.split(","):
            m = m.strip()
            arr = re.match(r"(\w+)\[(\d+)\]", m)
            members += [arr.group(1)] * int(arr.group(2)) if arr else [m]
    return members


def test_struct_layouts_match_header(lib_built):
    from sparse_matrix_algorithms_b200 import _lib as L

    for cname, pyst in [("sma_cheb_opts", L.ChebOpts), ("sma_polfed_opts", L.PolfedOpts),
                        ("sma_stats", L.Stats)]:
        members = _header_struct_members(cname)
        assert ctypes.sizeof(pyst) == 8 * len(members), cname
        named = [m for m in dict.fromkeys(members) if m != "reserved"]
        assert [f for f, _ in pyst._fields_ if f != "reserved"] == named, cname
    o = L.ChebOpts()
    L.load().sma_cheb_opts_default(ctypes.byref(o))
    assert (o.m0, o.degree, o.maxiter, o.tol, o.res_gate, o.seed) == (200, 80, 8, 1e-10, 1e-6, 1)
    p = L.PolfedOpts()
    L.load().sma_polfed_opts_default(ctypes.byref(p))
    assert (p.s, p.overextract, p.refine, p.mmax, p.rtol, p.extra_keep, p.chunk) == (8, 2, 1, 0, 1e-12, 8, 64)
    assert p.emin == -np.inf and p.emax == np.inf


def test_abi_version(lib_built):
    from sparse_matrix_algorithms_b200 import _lib as L

    assert L.load().sma_abi_version() == 1


@pytest.mark.parametrize("K", [0, 1, 3, 64, 777])
def test_coefficients_match_oracle(lib_built, K):
    import sparse_matrix_algorithms_b200 as S

    assert np.array_equal(S.jackson_kernel(K), O.jackson_kernel(K))
    for sh in [-1.5, -0.3, 0.0, 0.91]:
        assert np.array_equal(S.cheb_delta_coeffs(sh, K), O.cheb_delta_coeffs(sh, K))
    for a, b in [(-0.2, 0.1), (0.5, -0.5), (-3.0, 3.0), (0.0, 0.0)]:
        for jk in [True, False]:
            assert np.array_equal(S.cheb_window_coeffs(a, b, K, jk), O.cheb_window_coeffs(a, b, K, jk))
    c1 = S.cheb_smooth_window_coeffs(-0.2, 0.1, K)
    c2 = O.cheb_smooth_window_coeffs(-0.2, 0.1, K)
    assert np.abs(c1 - c2).max() < 1e-15  # same quadrature, summation order differs
    for w in ["step", "delta", "smooth"]:
        b1 = S.build_coeffs(K, -2.0, 6.0, 1.0, 0.5, 1.5, w)
        b2 = O.build_coeffs(K, -2.0, 6.0, 1.0, 0.5, 1.5, w)
        assert np.abs(b1 - b2).max() < 1e-15


def test_unknown_window_raises(lib_built):
    import sparse_matrix_algorithms_b200 as S

    with pytest.raises(S.ArgumentError, match="Unknown window type"):
        S.build_coeffs(10, 0.0, 4.0, 2.0, 1.0, 3.0, "boxcar")


def test_compute_calls_fail_loudly_without_a_gpu(lib_built):
    """No silent CPU path: without a usable device the context cannot be created."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import matrices as M

    with pytest.raises(S.SMAError):
        S.chebyshev_poly_real_symm_sparse(M.lap1d(50), 1.0, 2.0, smin=0.0, smax=4.0)


def test_host_closures_are_rejected(lib_built):
    import sparse_matrix_algorithms_b200 as S

    def matvec(y, x):
        y[:] = x

    with pytest.raises(S.ArgumentError, match="device"):
        S.MatrixFreeRealSymOp(10, matvec)
