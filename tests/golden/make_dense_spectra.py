"""Exact (dense LAPACK FP64) spectra of the configuration matrices that fit in host RAM.

Writes ``<name>_spectrum.npz`` next to this script with
  ``lam_min``, ``lam_max``  extreme eigenvalues,
  ``central``               the ``keep`` eigenvalues nearest (lam_min+lam_max)/2, ascending,
  ``central_first_index``   0-based index of ``central[0]`` in the full ascending spectrum,
  ``n``                     matrix order.
These are the count/accuracy oracle for the solver parity tests: the reference's own
test strategy compares against an exactly known spectrum (the 1D Laplacian,
``chebyshev_subspace_iteration.jl:903``), and for the Anderson/XXZ matrices the exact
spectrum is a dense symmetric eigensolve (dsyevd through scipy).

Usage:  python tests/golden/make_dense_spectra.py anderson_L20 [xxz_L18 ...]
The XXZ L=18 matrix (n=48620) needs ~19 GB of RAM and tens of minutes of CPU.
"""
import os
import sys
import time

import numpy as np
import scipy.linalg as sla

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from sparse_matrix_algorithms_b200.matrices import config_matrix  # noqa: E402


def main(names, keep=4000):
    for name in names:
        A = config_matrix(name)
        n = A.shape[0]
        t0 = time.time()
        D = A.toarray(order="F")
        lam = sla.eigh(D, eigvals_only=True, overwrite_a=True, check_finite=False, driver="evd")
        del D
        lam = np.sort(lam)
        c = 0.5 * (lam[0] + lam[-1])
        order = np.argsort(np.abs(lam - c), kind="stable")[: min(keep, n)]
        first = int(order.min())
        last = int(order.max())
        central = lam[first:last + 1]
        out = os.path.join(HERE, f"{name}_spectrum.npz")
        np.savez(out, lam_min=lam[0], lam_max=lam[-1], central=central,
                 central_first_index=first, n=n)
        print(f"{name}: n={n} [{lam[0]:.15g}, {lam[-1]:.15g}] kept {central.size} "
              f"central eigenvalues, {time.time() - t0:.1f} s -> {out}", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["anderson_L20"])
