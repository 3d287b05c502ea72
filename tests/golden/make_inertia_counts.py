"""Exact eigenvalue counts below given shifts by Sylvester's law of inertia.

For a real symmetric A and a shift s, a symmetric factorization
P (A - s I) P^T = L D L^T (L unit lower triangular) has as many negative entries in D as
A has eigenvalues below s.  SuperLU (scipy ``splu``) in symmetric mode with diagonal
pivoting only (``diag_pivot_thresh=0``, symmetric minimum-degree ordering) produces
P (A - s I) P^T = L U with U = D L^T whenever it keeps the diagonal pivots, which is
checked (row permutation equal to the column permutation); the count is then the number
of negative diagonal entries of U.  No polynomial filter or iterative eigensolver is
involved, so the counts are independent of the solvers under test.  FP64 on the host.

Usage:  python tests/golden/make_inertia_counts.py anderson_L64 --shifts -0.016975627263859053 0.016979915488252416
writes ``<name>_inertia.json`` next to this script: {shift: count below shift}.
"""
import argparse
import json
import os
import sys
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def count_below(A, shift: float) -> int:
    n = A.shape[0]
    M = (sp.csc_matrix(A) - shift * sp.identity(n, format="csc")).tocsc()
    lu = spla.splu(M, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                   options=dict(SymmetricMode=True))
    if not np.array_equal(lu.perm_r, lu.perm_c):
        raise RuntimeError("SuperLU left the diagonal: the factorization is not a congruence")
    d = lu.U.diagonal()
    if np.any(d == 0.0):
        raise RuntimeError("zero pivot: the shift is an eigenvalue to working precision")
    return int(np.count_nonzero(d < 0.0))


def main():
    from sparse_matrix_algorithms_b200.matrices import config_matrix

    ap = argparse.ArgumentParser()
    ap.add_argument("name")
    ap.add_argument("--shifts", type=float, nargs="+", required=True)
    a = ap.parse_args()
    A = config_matrix(a.name)
    out = {}
    for s in a.shifts:
        t0 = time.time()
        out[repr(s)] = count_below(A, s)
        print(f"{a.name}: {out[repr(s)]} eigenvalues below {s!r} ({time.time() - t0:.1f} s)", flush=True)
    path = os.path.join(HERE, f"{a.name}_inertia.json")
    old = json.load(open(path)) if os.path.exists(path) else {}
    old.update(out)
    json.dump(old, open(path, "w"), indent=1)


if __name__ == "__main__":
    main()
