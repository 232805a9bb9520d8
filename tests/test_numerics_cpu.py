"""Host-side numerics shared by the oracle and the device: the fixed
summation tree and the 2x2 minimum-norm solve."""
import numpy as np
import pytest

from oracle import pyoracle


@pytest.mark.parametrize("count", [0, 1, 7, 4096, 4097, 100_000, 1 << 20])
def test_tree_sum_exact_on_integers(count):
    v = np.arange(count, dtype=np.float64) % 97
    assert pyoracle.tree_sum(v) == float(v.sum())


def test_tree_sum_is_deterministic_and_accurate():
    rng = np.random.default_rng(0)
    v = rng.standard_normal(300_000)
    a = pyoracle.tree_sum(v)
    assert a == pyoracle.tree_sum(v.copy())
    assert abs(a - np.sum(v.astype(np.longdouble))) < 1e-10


@pytest.mark.parametrize("matrix,rhs", [
    ([[4.0, 1.0], [1.0, 3.0]], [1.0, 2.0]),
    ([[2.0, 1e-3], [1e-3, 5.0]], [-1.0, 0.5]),
    ([[1e-8, 2e-9], [2e-9, 3.0]], [1.0, 1.0]),
])
def test_solve_2x2_full_rank(matrix, rhs):
    got = pyoracle.solve_2x2(matrix, rhs)
    want = np.linalg.solve(np.array(matrix), np.array(rhs))
    assert np.allclose(got, want, rtol=1e-10, atol=0)


def test_solve_2x2_rank_deficient_is_minimum_norm_of_scaled_system():
    # sparse_operations.cpp:58-73 scales by D = diag(1/sqrt|m_ii|) and takes the
    # minimum-norm solution of D m D y = D rhs, then x = D y
    m = np.array([[1.0, 2.0], [2.0, 4.0]])
    rhs = np.array([1.0, 2.0])
    d = np.diag(1.0 / np.sqrt(np.abs(np.diag(m))))
    want = d @ np.linalg.pinv(d @ m @ d) @ (d @ rhs)
    got = pyoracle.solve_2x2(m, rhs)
    assert np.allclose(got, want, rtol=1e-12)


def test_solve_2x2_degenerate_inputs():
    assert np.array_equal(pyoracle.solve_2x2(np.zeros((2, 2)), [1.0, 1.0]), [0.0, 0.0])
    assert np.array_equal(pyoracle.solve_2x2([[np.nan, 0], [0, 1]], [1.0, 1.0]), [0.0, 0.0])
    assert np.array_equal(pyoracle.solve_2x2([[1.0, 0], [0, 1]], [np.inf, 1.0]), [0.0, 0.0])


def test_diffusion_batch_is_seeded_and_spd():
    from scipy import sparse

    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import problems
    a = problems.diffusion_batch(count=12, seed=5, n_min=200, n_max=3000)
    b = problems.diffusion_batch(count=12, seed=5, n_min=200, n_max=3000)
    assert len(a) == 12
    for x, y in zip(a, b):
        assert (x != y).nnz == 0 and x.shape == y.shape
        n = x.shape[0]
        assert 100 <= n <= 4000  # rounded grid sides around [n_min, n_max]
        assert abs(x - x.T).max() == 0.0
        # diagonally dominant with a positive diagonal: symmetric positive definite
        off = np.asarray(abs(x).sum(axis=1)).ravel() - np.abs(x.diagonal())
        assert np.all(x.diagonal() > off)
        assert x.has_sorted_indices and isinstance(x, sparse.csc_matrix)
    # both grid kinds appear (5-point rows hold at most 5 entries, 7-point up to 7)
    widths = {int(np.diff(x.indptr).max()) for x in a}
    assert widths & {5} and widths & {7}
