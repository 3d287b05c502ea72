"""Eigenvalues nearest a target energy for configuration matrices too large for a dense solve.

Shift-invert Lanczos (scipy ``eigsh`` with ``sigma``: ARPACK on (A - sigma I)^-1 through a
SuperLU factorisation), all in FP64 on the host. This is independent of the filtered
solvers under test: no Chebyshev polynomial is involved. Writes ``<name>_near<E>.npz``
next to this script with
  ``target``   the target energy,
  ``near``     the ``keep`` eigenvalues nearest ``target``, ascending,
  ``n``        matrix order.

Usage:  python tests/golden/make_shift_invert_spectra.py anderson_L64 [--keep 640] [--target 0]
The Anderson L=64 matrix (n=262144) takes a few minutes and a few GB of RAM.
"""
import argparse
import os
import sys
import time

import numpy as np
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from sparse_matrix_algorithms_b200.matrices import config_matrix  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="+")
    ap.add_argument("--keep", type=int, default=640)
    ap.add_argument("--target", type=float, default=0.0)
    a = ap.parse_args()
    for name in a.names:
        A = config_matrix(name).tocsc()
        n = A.shape[0]
        t0 = time.time()
        lam = spla.eigsh(A, k=a.keep, sigma=a.target, which="LM", return_eigenvectors=False,
                         tol=0.0, ncv=min(n, 2 * a.keep + 64))
        lam = np.sort(lam)
        tag = f"{a.target:g}".replace("-", "m").replace(".", "p")
        out = os.path.join(HERE, f"{name}_near{tag}.npz")
        np.savez(out, target=a.target, near=lam, n=n)
        print(f"{name}: n={n} kept {lam.size} eigenvalues in [{lam[0]:.15g}, {lam[-1]:.15g}] "
              f"near {a.target:g}, {time.time() - t0:.1f} s -> {out}", flush=True)


if __name__ == "__main__":
    main()
