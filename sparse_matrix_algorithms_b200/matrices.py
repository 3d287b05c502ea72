"""Seeded generators for the sparse real symmetric test matrices.

The reference ships exactly one fixture family, the 1D Laplacian
tridiag(-1, 2, -1) (``polfed.jl:1192-1195``, ``chebyshev_subspace_iteration.jl:875-879``)
with its analytic spectrum 2 - 2cos(k*pi/(n+1)) (``polfed.jl:1220-1222``).  The
workloads the solvers are measured on -- the 3D Anderson model and the random-field
XXZ spin chain in the Sz=0 sector -- have no generator in the reference, so they are
defined here, together with a documented counter-based random number generator so
that any other implementation (a Julia run elsewhere included) can rebuild the exact
same matrices bit for bit, or read them from the binary CSR files written by
:func:`save_csr`.

Random numbers
--------------
SplitMix64 (G. Steele, D. Lea, C. Flood, "Fast splittable pseudorandom number
generators", OOPSLA 2014) in counter form: draw ``k`` (k = 0, 1, ...) of stream
``seed`` is ``mix64(seed + (k + 1) * 0x9E3779B97F4A7C15 mod 2^64)`` and the uniform
double is ``(x >> 11) * 2^-53`` in [0, 1).  The same formula runs on the GPU for the
random start blocks (``sma_randn`` in the CUDA library).

All matrices are returned as ``scipy.sparse.csr_matrix`` (float64, int32 indices,
sorted columns, no duplicates).  A symmetric matrix's CSR arrays are identical to its
CSC arrays, which is what a Julia ``SparseMatrixCSC`` holds.
"""
from __future__ import annotations

import math
import struct

import numpy as np
import scipy.sparse as sp

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def mix64(z: np.ndarray) -> np.ndarray:
    """SplitMix64 output function on a uint64 array (wrapping arithmetic)."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def splitmix_uniform(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """Uniform doubles in [0, 1): draws ``offset .. offset+count-1`` of stream ``seed``."""
    k = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        ctr = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * GOLDEN
    x = mix64(ctr)
    return (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def splitmix_rademacher(seed: int, n: int, m: int) -> np.ndarray:
    """+-1 n x m block (column-major draw order): element (i, j), flat index k = i + j*n,
    is -1 when the top bit of draw k of stream ``seed ^ 0x2545F4914F6CDD1D`` is set.  The
    CUDA library's KPM start block uses the same rule."""
    s = np.uint64((seed ^ 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF)
    k = np.arange(1, n * m + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = mix64(s + k * GOLDEN)
    z = np.where((x >> np.uint64(63)) != 0, -1.0, 1.0)
    return z.reshape((m, n)).T.copy(order="F")


def splitmix_normal(seed: int, n: int, m: int) -> np.ndarray:
    """Standard normal n x m block (column-major draw order, like ``randn(n, m)``).

    Element (i, j) has flat index k = i + j*n and uses uniforms 2k and 2k+1 of stream
    ``seed ^ 0x5DEECE66D`` in the Box-Muller transform
    z = sqrt(-2 ln(1 - u0)) * cos(2 pi u1).  The CUDA library's ``sma_randn`` kernel
    evaluates the same formula (its transcendental functions may differ in the last
    bit).
    """
    s = (seed ^ 0x5DEECE66D) & 0xFFFFFFFFFFFFFFFF
    u = splitmix_uniform(s, 2 * n * m)
    u0 = u[0::2]
    u1 = u[1::2]
    z = np.sqrt(-2.0 * np.log1p(-u0)) * np.cos(2.0 * math.pi * u1)
    return z.reshape((m, n)).T.copy(order="F")


# --------------------------------------------------------------------------------------
# 1D Laplacian (the reference's own fixture)
# --------------------------------------------------------------------------------------

def lap1d(n: int) -> sp.csr_matrix:
    """tridiag(-1, 2, -1), as in ``polfed.jl:1192-1195`` / ``chebyshev_subspace_iteration.jl:875-879``."""
    e = np.ones(n - 1)
    A = sp.diags([-e, 2.0 * np.ones(n), -e], [-1, 0, 1], format="csr")
    return _canonical(A)


def lap1d_exact_eigs(n: int) -> np.ndarray:
    """Analytic spectrum 2 - 2cos(j pi/(n+1)), j=1..n, ascending (``polfed.jl:1220-1222``)."""
    j = np.arange(1, n + 1, dtype=np.float64)
    return 2.0 - 2.0 * np.cos(j * np.pi / (n + 1))


def lap1d_target_window(n: int, nev: int):
    """Window of ``nev`` central eigenvalues (``polfed.jl:1223-1233``).

    Returns ``(lam_exact, i1, i2, emin, emax, sigma)`` with 1-based ``i1, i2`` as in
    the reference.
    """
    lam = lap1d_exact_eigs(n)
    mid = min(max(_julia_round(n / 2), 1), n)
    i1 = min(max(mid - nev // 2, 1), n)
    i2 = min(max(i1 + nev - 1, 1), n)
    i1 = min(max(i2 - nev + 1, 1), n)
    emin = lam[i1 - 1]
    emax = lam[i2 - 1]
    return lam, i1, i2, emin, emax, 0.5 * (emin + emax)


def lap1d_interval_by_count(n: int, nev_target: int, center_frac: float = 0.5, pad: int = 2):
    """Padded window (``chebyshev_subspace_iteration.jl:980-992``).

    Returns ``(emin, emax, sigma, lam_ref, (i1, i2))`` with 1-based ``i1, i2``.
    """
    lam = lap1d_exact_eigs(n)
    ic = min(max(_julia_round(center_frac * n), 1), n)
    h = nev_target // 2
    i1 = max(1, ic - h)
    i2 = min(n, i1 + nev_target - 1)
    i1 = max(1, i2 - nev_target + 1)
    emin = lam[max(1, i1 - pad) - 1]
    emax = lam[min(n, i2 + pad) - 1]
    sigma = 0.5 * (lam[i1 - 1] + lam[i2 - 1])
    return emin, emax, sigma, lam[i1 - 1:i2].copy(), (i1, i2)


def _julia_round(x: float) -> int:
    """Julia's ``round(Int, x)``: round half to even (same as Python's ``round``)."""
    return int(round(x))


# --------------------------------------------------------------------------------------
# 3D Anderson model
# --------------------------------------------------------------------------------------

def anderson3d(L: int, W: float, seed: int, t: float = -1.0) -> sp.csr_matrix:
    """3D Anderson Hamiltonian on an L^3 periodic cubic lattice.

    H = sum_i eps_i |i><i| + t sum_<ij> |i><j|, t = -1 (nearest-neighbour hopping),
    eps_i = W * (u_i - 1/2) with u_i draw i of SplitMix64 stream ``seed``
    (i = x + L*y + L^2*z).  7 nonzeros per row for L >= 3.
    """
    n = L ** 3
    eps = W * (splitmix_uniform(seed, n) - 0.5)
    idx = np.arange(n, dtype=np.int64)
    x = idx % L
    y = (idx // L) % L
    z = idx // (L * L)
    rows = [idx]
    cols = [idx]
    vals = [eps]
    for dx, dy, dz in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        j = ((x + dx) % L) + L * ((y + dy) % L) + L * L * ((z + dz) % L)
        rows.append(idx)
        cols.append(j)
        vals.append(np.full(n, t))
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return _canonical(A.tocsr())


# --------------------------------------------------------------------------------------
# random-field XXZ chain, Sz = 0 sector
# --------------------------------------------------------------------------------------

def xxz_sz0_basis(L: int) -> np.ndarray:
    """Sz=0 basis: all L-bit integers with L/2 set bits, ascending.

    Bit i of a state is site i (1 = spin up).  The position of a state in this array
    is its basis index (lexicographic / combinatorial ranking).
    """
    if L % 2:
        raise ValueError("Sz=0 sector needs an even chain length")
    allst = np.arange(1 << L, dtype=np.int64)
    pc = np.zeros(1 << L, dtype=np.int64)
    for b in range(L):
        pc += (allst >> b) & 1
    return allst[pc == L // 2]


def xxz_sz0(L: int, h: float, seed: int, J: float = 1.0, Delta: float = 1.0) -> sp.csr_matrix:
    """Random-field XXZ spin-1/2 chain, periodic, restricted to Sz = 0.

    H = J sum_i (S^x_i S^x_{i+1} + S^y_i S^y_{i+1} + Delta S^z_i S^z_{i+1}) + sum_i h_i S^z_i
    with S = sigma/2, site L identified with site 0, and h_i = h * (2 u_i - 1),
    u_i draw i (i = 0..L-1) of SplitMix64 stream ``seed``.  In the S^z basis the
    diagonal is J*Delta*sum s_i s_{i+1} + sum h_i s_i (s = +-1/2) and every
    antiparallel bond couples to the bond-flipped state with amplitude J/2.
    """
    hfield = h * (2.0 * splitmix_uniform(seed, L) - 1.0)
    states = xxz_sz0_basis(L)
    n = states.size
    rank = np.full(1 << L, -1, dtype=np.int64)
    rank[states] = np.arange(n, dtype=np.int64)
    sz = np.empty((L, n))
    for i in range(L):
        sz[i] = np.where((states >> i) & 1, 0.5, -0.5)
    diag = np.zeros(n)
    for i in range(L):
        j = (i + 1) % L
        diag += J * Delta * sz[i] * sz[j]
        diag += hfield[i] * sz[i]
    rows = [np.arange(n, dtype=np.int64)]
    cols = [np.arange(n, dtype=np.int64)]
    vals = [diag]
    for i in range(L):
        j = (i + 1) % L
        bi = (states >> i) & 1
        bj = (states >> j) & 1
        m = bi != bj
        flipped = states[m] ^ ((1 << i) | (1 << j))
        rows.append(np.nonzero(m)[0])
        cols.append(rank[flipped])
        vals.append(np.full(int(m.sum()), 0.5 * J))
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return _canonical(A.tocsr())


# --------------------------------------------------------------------------------------
# helpers
# --------------------------------------------------------------------------------------

def _canonical(A: sp.spmatrix) -> sp.csr_matrix:
    A = sp.csr_matrix(A, dtype=np.float64)
    A.sum_duplicates()
    A.sort_indices()
    idx = np.int32 if A.nnz < 2**31 - 1 else np.int64  # scipy wants one index dtype
    A.indices = A.indices.astype(idx)
    A.indptr = A.indptr.astype(idx)
    return A


def save_csr(path: str, A: sp.csr_matrix) -> None:
    """Write ``A`` as a little-endian binary CSR file.

    Layout: magic ``b"SMACSR01"``, int64 n, int64 nnz, then int64 rowptr[n+1]
    (0-based), int32 colind[nnz], float64 values[nnz].
    """
    A = _canonical(A)
    n = A.shape[0]
    with open(path, "wb") as f:
        f.write(b"SMACSR01")
        f.write(struct.pack("<qq", n, A.nnz))
        f.write(A.indptr.astype("<i8").tobytes())
        f.write(A.indices.astype("<i4").tobytes())
        f.write(A.data.astype("<f8").tobytes())


def load_csr(path: str) -> sp.csr_matrix:
    """Read a file written by :func:`save_csr`."""
    with open(path, "rb") as f:
        if f.read(8) != b"SMACSR01":
            raise ValueError(f"{path}: not an SMACSR01 file")
        n, nnz = struct.unpack("<qq", f.read(16))
        indptr = np.frombuffer(f.read(8 * (n + 1)), dtype="<i8")
        indices = np.frombuffer(f.read(4 * nnz), dtype="<i4")
        data = np.frombuffer(f.read(8 * nnz), dtype="<f8")
    return _canonical(sp.csr_matrix((data, indices, indptr), shape=(n, n)))


def save_mtx(path: str, A: sp.spmatrix, comment: str = "") -> None:
    """Write ``A`` in Matrix Market coordinate format: ``real symmetric`` (lower triangle,
    1-based) when A == A^T, ``real general`` otherwise; values with 17 significant digits so
    that a reader recovers every double exactly.  Julia reads it with
    ``MatrixMarket.mmread``."""
    A = _canonical(A)
    n = A.shape[0]
    sym = (abs(A - A.T)).nnz == 0
    C = sp.tril(A).tocoo() if sym else A.tocoo()
    order = np.lexsort((C.row, C.col))  # column-major entry order
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {'symmetric' if sym else 'general'}\n")
        for line in comment.splitlines():
            f.write(f"% {line}\n")
        f.write(f"{n} {A.shape[1]} {C.nnz}\n")
        for i, j, v in zip(C.row[order], C.col[order], C.data[order]):
            f.write(f"{i + 1} {j + 1} {float(v)!r}\n")  # shortest round-trip repr


def load_mtx(path: str) -> sp.csr_matrix:
    """Read a Matrix Market coordinate file (``real``/``integer``, ``general`` or
    ``symmetric``) into the canonical CSR form."""
    with open(path) as f:
        header = f.readline().split()
        if len(header) < 5 or header[0] != "%%MatrixMarket" or header[2] != "coordinate":
            raise ValueError(f"{path}: not a Matrix Market coordinate file")
        symmetric = header[4].lower() == "symmetric"
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, nnz = (int(x) for x in line.split())
        data = np.loadtxt(f, ndmin=2) if nnz else np.zeros((0, 3))
    i = data[:, 0].astype(np.int64) - 1
    j = data[:, 1].astype(np.int64) - 1
    v = data[:, 2].astype(np.float64)
    if symmetric:
        off = i != j
        i, j, v = np.concatenate([i, j[off]]), np.concatenate([j, i[off]]), np.concatenate([v, v[off]])
    return _canonical(sp.coo_matrix((v, (i, j)), shape=(m, n)).tocsr())


def config_matrix(name: str) -> sp.csr_matrix:
    """The matrices of the benchmark configurations, by name.

    ``anderson_L20``  3D Anderson L=20 (n=8000), W=16.5, seed 0
    ``xxz_L18``       XXZ L=18 Sz=0 (n=48620), h=5, seed 1
    ``anderson_L64``  3D Anderson L=64 (n=262144), W=16.5, seed 2
    ``xxz_L20``       XXZ L=20 Sz=0 (n=184756), h=3, seed 3
    ``anderson_L96``  3D Anderson L=96 (n=884736), W=12, seed 4
    """
    table = {
        "anderson_L20": lambda: anderson3d(20, 16.5, 0),
        "xxz_L18": lambda: xxz_sz0(18, 5.0, 1),
        "anderson_L64": lambda: anderson3d(64, 16.5, 2),
        "xxz_L20": lambda: xxz_sz0(20, 3.0, 3),
        "anderson_L96": lambda: anderson3d(96, 12.0, 4),
    }
    if name not in table:
        raise KeyError(f"unknown configuration matrix {name!r}; known: {sorted(table)}")
    return table[name]()
