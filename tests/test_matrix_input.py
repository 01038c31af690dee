"""Host logic of the assembled-matrix input (CPU): the union pattern of K, M and D,
the scatter of each matrix onto it, and the (slave, master) pairs read from the
reference's fold operators (saw3d/bc_solve.py:25-33)."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import hex27 as oh
from sawsim_b200.engine import _canonical, _fold_pairs, _on_pattern, _union_pattern


def _rand(n, density, seed):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=rng, format='coo')
    return sp.coo_matrix((A.data + 1j * rng.standard_normal(A.nnz), (A.row, A.col)), shape=(n, n))


def test_union_pattern_and_scatter():
    n = 40
    K, M = _rand(n, 0.1, 1), _rand(n, 0.05, 2)
    Kc, Mc = _canonical(K, n), _canonical(M, n)
    indptr, indices, keys = _union_pattern([Kc, Mc])
    U = sp.csr_matrix((np.ones(indices.size), indices, indptr), shape=(n, n))
    assert U.has_sorted_indices
    assert set(zip(*U.nonzero())) == set(zip(*Kc.nonzero())) | set(zip(*Mc.nonzero()))
    for A, Ac in ((K, Kc), (M, Mc)):
        v = _on_pattern(Ac, keys)
        B = sp.csr_matrix((v, indices, indptr), shape=(n, n))
        assert abs(B - A.tocsr()).max() == 0


def test_duplicates_summed_and_explicit_zeros_kept():
    n = 4
    A = sp.coo_matrix((np.array([1.0, 2.0, 0.0, 3.0]), (np.array([0, 0, 1, 2]), np.array([1, 1, 2, 3]))),
                      shape=(n, n))
    Ac = _canonical(A, n)
    assert Ac.nnz == 3                       # (0,1) summed, the explicit zero (1,2) kept
    assert Ac[0, 1] == 3.0
    _, _, keys = _union_pattern([Ac])
    assert 1 * n + 2 in keys


def test_entries_outside_pattern_rejected():
    n = 10
    K = _canonical(sp.eye(n), n)
    _, _, keys = _union_pattern([K])
    with pytest.raises(ValueError):
        _on_pattern(_canonical(sp.eye(n, k=1), n), keys)
    with pytest.raises(ValueError):
        _canonical(sp.eye(n + 1), n)


def test_fold_pairs_read_the_reference_operator():
    gdof = 12
    slaves, masters = np.array([3, 7, 11]), np.array([0, 4, 8])
    T = oh._fold(slaves, masters, gdof)
    s, m = _fold_pairs(T)
    assert np.array_equal(s, slaves) and np.array_equal(m, masters)
