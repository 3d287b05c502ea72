"""The divided difference behind the MIXED POLFED polish (sma_divided_difference, host
code): for p = sum c_m T_m and a shift t, (p(s) - p(t)) / (s - t) = sum e_m T_m(s).  Checked
against the oracle's Chebyshev-series long division and against the defining identity at
sample points.  No GPU needed."""
import numpy as np
import pytest
from numpy.polynomial import chebyshev as C

import sma_oracle as O


def _lib_dd(c, t):
    from sparse_matrix_algorithms_b200 import _lib as L

    c = np.ascontiguousarray(c, dtype=np.float64)
    e = np.zeros(len(c) - 1)
    pt = np.zeros(1)
    L.check(L.load().sma_divided_difference(c.ctypes.data, len(c) - 1, float(t), e.ctypes.data,
                                            pt.ctypes.data))
    return e, float(pt[0])


@pytest.mark.parametrize("K", [1, 2, 7, 120, 1200])
@pytest.mark.parametrize("window", ["step", "delta"])
def test_divided_difference_matches_oracle(lib_built, K, window):
    c = O.build_coeffs(K, -12.0, 12.0, 0.01, -0.02, 0.04, window, window == "delta")
    scale = np.abs(c).sum()
    for t in [-0.9, -1e-3, 0.0, 0.0017, 0.5]:
        e, pt = _lib_dd(c, t)
        e_o, pt_o = O.divided_difference(c, t)
        assert abs(pt - pt_o) <= 1e-13 * scale
        assert np.abs(e - e_o).max() <= 1e-11 * max(1.0, np.abs(e_o).max())
        s = np.linspace(-1, 1, 41)
        lhs = C.chebval(s, c) - pt
        rhs = (s - t) * C.chebval(s, e)
        assert np.abs(lhs - rhs).max() <= 1e-11 * max(1.0, np.abs(e).sum())


def test_divided_difference_rejects_degree_zero(lib_built):
    from sparse_matrix_algorithms_b200 import _lib as L

    c = np.ones(1)
    e = np.zeros(1)
    pt = np.zeros(1)
    rc = L.load().sma_divided_difference(c.ctypes.data, 0, 0.0, e.ctypes.data, pt.ctypes.data)
    assert rc == L.SMA_ERR_ARG
