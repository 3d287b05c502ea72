"""Host-side planning logic without a GPU: KPM window placement (the library's kpm_count is
host code) on moments from the KPM oracle, the plain rules, and the benchmark's host
Gershgorin bounds."""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import sma_oracle as O  # noqa: E402
from sparse_matrix_algorithms_b200 import matrices as M  # noqa: E402
from sparse_matrix_algorithms_b200 import planner as P  # noqa: E402


def test_windows_by_count_track_dense_counts(lib_built):
    A = M.anderson3d(10, 16.5, 0)
    lam = np.linalg.eigvalsh(A.toarray())
    smin, smax = O.gershgorin_bounds(A)
    mu = O.kpm_moments(A, 256, 32, 11, smin, smax)
    wins = P.windows_by_count(mu, A.shape[0], smin, smax, 0.0, [40, 60, 30])
    for (a, b), want in zip(wins, [40, 60, 30]):
        got = int(np.sum((lam >= a) & (lam <= b)))
        assert abs(got - want) <= 0.2 * want + 4, (a, b, got, want)
    # contiguous, increasing, and centred on the requested energy
    assert all(wins[i][1] == wins[i + 1][0] for i in range(2))
    assert wins[0][0] < 0.0 < wins[-1][1]


def test_polfed_plain_rule_and_nev():
    K, mmax = P.polfed_plain_rule(100.0, -10.0, 10.0, -0.5, 0.5, 16)
    assert K == math.ceil(12 * 10.0 / 1.0) and mmax == math.ceil(2.8 * 100 / 16)
    assert P.polfed_nev(49.6) == 62 and P.polfed_nev(0.0) == 4
    assert P.polfed_cost(100, 10, 8) == 8000


def test_bench_host_gershgorin_matches_oracle():
    import bench

    for A in (M.anderson3d(8, 16.5, 1), M.xxz_sz0(10, 3.0, 2)):
        lo, hi = bench.host_gershgorin(A)
        lo2, hi2 = O.gershgorin_bounds(A)
        assert abs(lo - lo2) <= 1e-12 * abs(lo2) and abs(hi - hi2) <= 1e-12 * abs(hi2)
