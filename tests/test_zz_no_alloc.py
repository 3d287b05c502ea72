"""The allocation-free filter entry point, sma_apply_poly_block_noalloc.

It exists for callers that cannot allocate device memory -- a process whose GPU memory
another allocator has already reserved, or a latency-critical loop that must not pay for
cudaMalloc/cudaFree -- and keeps its recurrence blocks in a static device array instead.
These tests call it through the C ABI and compare it with the regular entry point,
sma_apply_poly_block_dev, on two calls in a row (the array keeps the previous call's
contents, which must not leak into the next result), within the FP64 tolerance of the
filter parity tests (1e-12 relative to the block's magnitude).  The file is named so that
pytest collects it last.
"""
import numpy as np
import pytest

import sma_oracle as O
from sparse_matrix_algorithms_b200 import matrices as M

pytestmark = pytest.mark.gpu


def _run(entry, op, c, smin, smax, Q, ldq, Y, ldy, b):
    import torch
    from sparse_matrix_algorithms_b200 import _lib as L

    torch.cuda.synchronize()
    fn = getattr(L.load(), entry)
    if entry == "sma_apply_poly_block_dev":
        rc = fn(op.handle, c.ctypes.data, len(c) - 1, smin, smax, Q.data_ptr(), ldq, Y.data_ptr(),
                ldy, b, 0)
    else:
        rc = fn(op.handle, c.ctypes.data, len(c) - 1, smin, smax, Q.data_ptr(), ldq, Y.data_ptr(),
                ldy, b)
    L.check(rc)
    return Y.cpu().numpy()


def test_noalloc_filter_matches_regular_entry_on_two_calls(lib_built):
    import torch
    import sparse_matrix_algorithms_b200 as S

    A = M.xxz_sz0(14, 5.0, 1)
    n = A.shape[0]
    op = S.SparseOperator(A)
    smin, smax = O.gershgorin_bounds(A)
    cases = [  # (width, leading dims, degree, window) -- the second call is narrower
        (24, 24, 24, 300, "step"),
        (10, 13, 12, 45, "delta"),
    ]
    for b, ldq, ldy, K, window in cases:
        c = np.ascontiguousarray(O.build_coeffs(K, smin, smax, 0.2, -0.5, 0.4, window, True))
        Qh = np.zeros((n, ldq))
        Qh[:, :b] = M.splitmix_normal(b + K, n, b)
        Q = torch.as_tensor(Qh, device="cuda")
        Yref = _run("sma_apply_poly_block_dev", op, c, smin, smax, Q, ldq,
                    torch.zeros((n, ldy), dtype=torch.float64, device="cuda"), ldy, b)
        Y = _run("sma_apply_poly_block_noalloc", op, c, smin, smax, Q, ldq,
                 torch.full((n, ldy), 3.0, dtype=torch.float64, device="cuda"), ldy, b)
        scale = max(np.abs(Yref[:, :b]).max(), np.abs(Qh).max())
        assert np.abs(Y[:, :b] - Yref[:, :b]).max() <= 1e-12 * scale
        assert np.all(Y[:, b:] == 3.0)  # columns beyond b untouched


@pytest.mark.parametrize("stencil", ["lap1d", "anderson", "xxz"])
def test_noalloc_filter_stencil_operators(lib_built, stencil):
    """Every model stencil the entry point accepts: 1D Laplacian, Anderson, XXZ."""
    import torch
    import sparse_matrix_algorithms_b200 as S

    if stencil == "lap1d":
        op, smin, smax = S.Lap1dOperator(5000), 0.0, 4.0
    elif stencil == "anderson":
        op = S.AndersonOperator(12, 16.5, 5)
        smin, smax = O.gershgorin_bounds(M.anderson3d(12, 16.5, 5))
    else:
        op = S.XXZOperator(12, 5.0, 1)
        smin, smax = O.gershgorin_bounds(M.xxz_sz0(12, 5.0, 1))
    n, b = op.n, 16
    mid = 0.5 * (smin + smax)
    c = np.ascontiguousarray(O.build_coeffs(80, smin, smax, mid, mid - 0.1, mid + 0.1, "delta", True))
    Q = torch.as_tensor(M.splitmix_normal(3, n, b), device="cuda").contiguous()
    for _ in range(2):
        Yref = _run("sma_apply_poly_block_dev", op, c, smin, smax, Q, b,
                    torch.empty((n, b), dtype=torch.float64, device="cuda"), b, b)
        Y = _run("sma_apply_poly_block_noalloc", op, c, smin, smax, Q, b,
                 torch.empty((n, b), dtype=torch.float64, device="cuda"), b, b)
        assert np.abs(Y - Yref).max() <= 1e-12 * max(1.0, np.abs(Yref).max())


def test_noalloc_filter_size_limit(lib_built):
    import torch
    import sparse_matrix_algorithms_b200 as S
    from sparse_matrix_algorithms_b200 import _lib as L

    b = 16
    c = np.ascontiguousarray(O.build_coeffs(80, 0.0, 4.0, 2.0, 1.9, 2.1, "delta", True))
    Q = torch.zeros((4, b), dtype=torch.float64, device="cuda")
    # n*b beyond the 2,097,152-element capacity is rejected before any launch
    big = S.Lap1dOperator(300_000)
    rc = L.load().sma_apply_poly_block_noalloc(big.handle, c.ctypes.data, len(c) - 1, 0.0, 4.0,
                                               Q.data_ptr(), b, Q.data_ptr(), b, b)
    assert rc == L.SMA_ERR_ARG
    assert b"capacity" in L.load().sma_last_error()
    # half storage needs an extra product block, so it is refused rather than allocated
    half = S.SparseOperator(M.lap1d(64), storage="upper")
    rc = L.load().sma_apply_poly_block_noalloc(half.handle, c.ctypes.data, len(c) - 1, 0.0, 4.0,
                                               Q.data_ptr(), b, Q.data_ptr(), b, b)
    assert rc == L.SMA_ERR_ARG
