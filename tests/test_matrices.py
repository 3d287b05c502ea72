"""The seeded generators: structure, symmetry, exact small cases, file round trip."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from sparse_matrix_algorithms_b200 import matrices as M


def test_splitmix_counter_stream_known_values():
    # SplitMix64 from state 0: first outputs of the published generator
    x = M.mix64(np.array([0x9E3779B97F4A7C15], dtype=np.uint64))
    assert int(x[0]) == 0xE220A8397B1DCDAF
    u = M.splitmix_uniform(7, 5)
    assert np.all((u >= 0) & (u < 1))
    assert np.array_equal(M.splitmix_uniform(7, 3, offset=2), u[2:])


def test_splitmix_normal_moments_and_layout():
    Z = M.splitmix_normal(1, 2000, 50)
    assert Z.shape == (2000, 50) and Z.flags.f_contiguous
    assert abs(Z.mean()) < 0.01 and abs(Z.std() - 1) < 0.01
    # column-major draw order: the first column equals the first n draws
    assert np.array_equal(M.splitmix_normal(1, 2000, 1)[:, 0], Z[:, 0])


def test_lap1d_and_its_spectrum():
    A = M.lap1d(60)
    assert A.nnz == 3 * 60 - 2
    assert np.allclose(np.linalg.eigvalsh(A.toarray()), M.lap1d_exact_eigs(60), atol=1e-13)


def test_anderson_structure():
    L = 6
    A = M.anderson3d(L, 16.5, 3)
    n = L ** 3
    assert A.shape == (n, n) and A.nnz == 7 * n
    assert (abs(A - A.T)).nnz == 0
    d = A.diagonal()
    assert np.all(np.abs(d) <= 16.5 / 2)
    off = A - sp.diags(d)
    assert np.all(off.data == -1.0)
    # neighbours of site 0: x+-1, y+-L, z+-L^2 (periodic)
    assert sorted(A[0].indices.tolist()) == sorted([0, 1, L - 1, L, L * (L - 1), L * L, L * L * (L - 1)])
    assert np.array_equal(A.diagonal(), 16.5 * (M.splitmix_uniform(3, n) - 0.5))


def _xxz_dense_kron(L, h, seed):
    sx = np.array([[0, 1], [1, 0]]) / 2
    sy = np.array([[0, -1j], [1j, 0]]) / 2
    sz = np.array([[1, 0], [0, -1]]) / 2

    def op(o, i):
        r = np.array([[1.0 + 0j]])
        for site in reversed(range(L)):  # bit i of the index is site i
            r = np.kron(r, o if site == i else np.eye(2))
        return r

    hf = h * (2 * M.splitmix_uniform(seed, L) - 1)
    H = sum(op(sx, i) @ op(sx, (i + 1) % L) + op(sy, i) @ op(sy, (i + 1) % L)
            + op(sz, i) @ op(sz, (i + 1) % L) for i in range(L))
    H = H + sum(hf[i] * op(sz, i) for i in range(L))
    return H.real


@pytest.mark.parametrize("L", [4, 6, 8])
def test_xxz_matches_kronecker_construction(L):
    A = M.xxz_sz0(L, 2.5, 11)
    H = _xxz_dense_kron(L, 2.5, 11)
    # Kronecker basis: bit = 0 is spin up (sz=+1/2); ours: bit = 1 is up
    idx = [(~s) & ((1 << L) - 1) for s in M.xxz_sz0_basis(L)]
    Hs = H[np.ix_(idx, idx)]
    assert np.allclose(Hs, A.toarray(), atol=1e-14)


def test_xxz_sizes_and_density():
    A = M.xxz_sz0(12, 5.0, 1)
    assert A.shape == (924, 924)
    assert (abs(A - A.T)).nnz == 0
    L = 12
    assert abs(A.nnz / A.shape[0] - (1 + L * L / (2 * (L - 1)))) < 1e-9


def test_matrix_market_round_trip_exact(tmp_path):
    for A in [M.xxz_sz0(8, 3.0, 2), M.anderson3d(4, 16.5, 1)]:
        p = os.path.join(tmp_path, "a.mtx")
        M.save_mtx(p, A, comment="test matrix")
        head = open(p).readline()
        assert head.strip() == "%%MatrixMarket matrix coordinate real symmetric"
        B = M.load_mtx(p)
        for arr in ("indptr", "indices", "data"):  # every double recovered exactly
            assert np.array_equal(getattr(A, arr), getattr(B, arr))
    G = M._canonical(sp.csr_matrix(np.array([[1.0, 2.0], [0.0, 3.0]])))
    p = os.path.join(tmp_path, "g.mtx")
    M.save_mtx(p, G)
    H = M.load_mtx(p)
    assert "general" in open(p).readline()
    assert np.array_equal(H.toarray(), G.toarray())


def test_csr_file_round_trip(tmp_path):
    A = M.anderson3d(5, 16.5, 2)
    p = os.path.join(tmp_path, "a.csr")
    M.save_csr(p, A)
    B = M.load_csr(p)
    assert (A != B).nnz == 0 and np.array_equal(A.indptr, B.indptr)
