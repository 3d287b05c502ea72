"""B200 (sm_100a) implementation of the solve-free interior eigensolvers of
MathiasTensor/sparse_matrix_algorithms: Chebyshev-filtered subspace iteration
(``chebyshev_poly_real_symm_sparse``) and POLFED (``polfed``).

The numerical work runs in ``libsma.so`` (CUDA, C ABI in ``include/sma.h``); this
package is its Python mirror of the reference's API plus the seeded test-matrix
generators.
"""
from .api import (  # noqa: F401
    AndersonOperator,
    ArgumentError,
    XXZOperator,
    Context,
    DeviceMatblock,
    Lap1dOperator,
    MatrixFreeRealSymOp,
    SMAError,
    SparseOperator,
    apply_poly_block,
    build_coeffs,
    cheb_delta_coeffs,
    cheb_smooth_window_coeffs,
    cheb_window_coeffs,
    chebyshev_poly_real_symm_sparse,
    context,
    gershgorin_bounds,
    jackson_kernel,
    kpm_count,
    kpm_moments,
    lanczos_bounds,
    polfed,
    polfed_windows,
    slice_spectrum,
)
from . import matrices  # noqa: F401
