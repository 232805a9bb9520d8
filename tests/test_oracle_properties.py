"""The reference's C++ property tests (tests/test.cpp) restated on the
oracle, in both summation orders."""
import numpy as np
import pytest
from scipy import sparse
from scipy.sparse.linalg import norm

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import problems
from tests.helpers import METHODS

N = 12
A = problems.tridiagonal(N)
I = sparse.identity(N, format="csc")
BASE = dict(M0=I, Pr=I, max_iterations=8, tolerance=1e-14, max_density=1.0)


def run(family, name, order=pyoracle.ORDER_REFERENCE, **kw):
    args = dict(BASE)
    args.update(kw)
    return pyoracle.run(family, name, A, order=order, **args)


def true_residual(M):
    return norm(sparse.identity(N) - A @ M)


@pytest.mark.parametrize("order", [pyoracle.ORDER_REFERENCE, pyoracle.ORDER_DEVICE])
@pytest.mark.parametrize("family,name", METHODS)
def test_thread_equivalence_and_decrease(family, name, order):
    # tests/test.cpp:30-39,61-81: 1 vs 2 column batches, monotone decrease
    one = run(family, name, order, num_threads=1)
    two = run(family, name, order, num_threads=2)
    initial = true_residual(I)
    for r in (one, two):
        assert len(r.history) == r.iterations + 1
        assert r.history[0]["iteration"] == 0 and r.history[-1]["iteration"] == r.iterations
        assert r.history[-1]["residual_norm"] < initial
    assert one.iterations == two.iterations
    assert norm(one.M - two.M) < 1e-10
    assert abs(one.history[-1]["residual_norm"] - two.history[-1]["residual_norm"]) < 1e-10


@pytest.mark.parametrize("family,name", METHODS)
def test_dropping_budget(family, name):
    # tests/test.cpp:41-48,84-90,141-151
    kw = dict(max_iterations=3, max_density=0.12, tolerance=0.0)
    one = run(family, name, num_threads=1, **kw)
    four = run(family, name, num_threads=4, **kw)
    budget = max(N, int(np.floor(0.12 * N * N)))
    for r in (one, four):
        assert r.M.nnz <= budget
        assert r.iterations == 3
    assert norm(one.M - four.M) < 1e-10


@pytest.mark.parametrize("family,name", METHODS)
def test_density_stop_without_dropping(family, name):
    # tests/test.cpp:50-59,153-165
    r = run(family, name, max_iterations=8, tolerance=0.0, max_density=0.2, enable_dropping=False)
    assert not r.converged and 0 < r.iterations < 8
    assert r.history[-1]["density_m"] >= 0.2


def test_absolute_stop():
    # tests/test.cpp:130-138
    tol = 0.9 * true_residual(I)
    r = run("global_spai", "mr", num_threads=2, tolerance=tol)
    assert r.converged and r.iterations == 1 and len(r.history) == 2
    assert r.history[-1]["residual_norm"] < tol


def test_reported_vs_true_residual():
    # tests/test.cpp:167-177
    r = run("inner_outer", "lomr", num_threads=2, max_iterations=20, tolerance=1e-20)
    assert r.iterations == 20 and not r.converged
    assert abs(r.history[-1]["residual_norm"] - true_residual(r.M)) < 1e-9


def test_topk_caps_columns():
    A2 = problems.laplacian_2d(10)
    r = pyoracle.run("global_spai", "mr", A2, M0=problems.diagonal_inverse(A2), max_iterations=5, tolerance=0.0,
                     max_density=0.05, topk_per_column=4)
    assert np.diff(r.M.indptr).max() <= 4
    assert np.all(r.M.diagonal() != 0)


def test_error_messages():
    with pytest.raises(RuntimeError, match="max_iterations must be positive"):
        run("global_spai", "mr", max_iterations=0)
    with pytest.raises(RuntimeError, match="max_density is too small"):
        run("global_spai", "mr", max_density=0.01)
    with pytest.raises(RuntimeError, match="Invalid threads count value"):
        run("global_spai", "mr", num_threads=0)
    with pytest.raises(RuntimeError, match="inner_iterations must be positive"):
        run("inner_outer", "mr", inner_iterations=0)
