"""Exact eigenvalue counts by Sylvester inertia (tests/golden/make_inertia_counts.py),
checked against dense spectra, and the committed count of the C3 window."""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
sys.path.insert(0, ROOT)

from make_inertia_counts import count_below  # noqa: E402
from sparse_matrix_algorithms_b200 import matrices as M  # noqa: E402


def test_inertia_counts_match_dense():
    for A in (M.anderson3d(9, 16.5, 3), M.xxz_sz0(12, 2.0, 4)):
        lam = np.linalg.eigvalsh(A.toarray())
        for s in np.quantile(lam, [0.05, 0.37, 0.5, 0.81]) + 1e-7:
            assert count_below(A, float(s)) == int(np.sum(lam < s))


def test_c3_window_count_fixture():
    """494 eigenvalues of the Anderson L=64 matrix lie in the benchmark's C3 window (the
    KPM placement aimed at 500)."""
    sys.path.insert(0, ROOT)
    import bench

    below = json.load(open(os.path.join(ROOT, "tests", "golden", "anderson_L64_inertia.json")))
    emin, emax = bench.C3_WINDOW
    assert below[repr(emax)] - below[repr(emin)] == 494
