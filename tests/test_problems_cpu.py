"""CPU tests of the synthetic problem generators behind the configurations
(pevsl_b200/problems.py): the matrices are what their docstrings say, so
that the benchmark and the tests measure the workloads they name."""
import numpy as np
import scipy.sparse as sp

from pevsl_b200.problems import (laplacian, laplacian_eigenvalues, laplacian_shifted,
                                 multi_laplacian_set, random_coef_laplacian,
                                 random_sparse_symmetric)


def as_sparse(n, ia, ja, a):
    return sp.csr_matrix((a, ja, ia), shape=(n, n))


def test_laplacian_matches_its_eigenvalues():
    n, ia, ja, a = laplacian(6, 5, 4)
    M = as_sparse(n, ia, ja, a).toarray()
    assert np.array_equal(M, M.T)
    w = np.linalg.eigvalsh(M)
    ex = laplacian_eigenvalues(6, 5, 4, 0.0, 100.0)
    assert len(ex) == n and np.max(np.abs(np.sort(w) - ex)) <= 1e-12 * ex[-1]
    assert int(ia[-1]) == 7 * n - 2 * (6 * 5 + 6 * 4 + 5 * 4)


def test_shifted_laplacian_moves_every_eigenvalue():
    n, ia, ja, a = laplacian_shifted(7, 7, 1, 0.25)
    w = np.linalg.eigvalsh(as_sparse(n, ia, ja, a).toarray())
    ex = laplacian_eigenvalues(7, 7, 1, 0.0, 100.0) + 0.25
    assert np.max(np.abs(np.sort(w) - ex)) <= 1e-12 * ex[-1]


def test_random_sparse_symmetric_shape():
    n, bw = 20000, 500
    n_, ia, ja, a = random_sparse_symmetric(n, 16, bw, 3)
    assert n_ == n
    M = as_sparse(n, ia, ja, a)
    assert (M - M.T).count_nonzero() == 0  # exactly symmetric
    rows = np.repeat(np.arange(n), np.diff(ia))
    assert np.max(np.abs(ja - rows)) <= bw  # offsets within the bandwidth
    lens = np.diff(ia)
    assert 14 <= lens.mean() <= 18
    # draws outside the matrix are dropped: no row collects them
    assert lens.max() <= 40
    assert np.all(np.diff(ja[ia[0]:ia[1]]) > 0)  # columns sorted
    d = M.diagonal()
    assert np.all((d > 3.0) & (d < 6.0))


def test_random_coefficient_laplacian_is_an_m_matrix():
    n, ia, ja, a = random_coef_laplacian(6, 5, 4, seed=2)
    M = as_sparse(n, ia, ja, a).toarray()
    assert np.array_equal(M, M.T)
    off = M - np.diag(np.diag(M))
    assert np.all(off <= 0.0) and np.all(off >= -2.0)
    # row sums: zero inside, the boundary edges' weights (>= 0.5) on the
    # boundary; irreducibly diagonally dominant, hence positive definite
    rs = np.diag(M) + off.sum(axis=1)
    assert np.all(rs >= -1e-12) and np.max(rs) >= 0.5
    assert np.linalg.eigvalsh(M)[0] > 0


def test_multi_laplacian_set_counts():
    P = multi_laplacian_set(count=4, seed=5, per_slice=20)
    assert len(P) == 4
    for p in P:
        assert 1e4 <= p["n"] <= 5e5 and 2 <= p["nslices"] <= 8
        ev = laplacian_eigenvalues(*p["grid"], 0.0, 100.0) + p["shift"]
        edges = np.array(p["intv"])
        counts = [int(np.sum((ev >= edges[k]) & (ev < edges[k + 1])))
                  for k in range(p["nslices"])]
        assert counts == p["counts"]
        assert abs(sum(counts) - 20 * p["nslices"]) <= 2 * p["nslices"]
        # slice ends away from every eigenvalue
        for e in edges:
            assert np.min(np.abs(ev - e)) > 1e-11
