"""The adjoint oracle against central finite differences (the math of the
device adjoints, checked on the CPU), and the adjoint entry points' input
checks, which run before any device work."""
import ctypes

import numpy as np
import pytest
from scipy import sparse
from scipy.sparse import linalg as splinalg

from oracle import adjoint_oracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib, adjoint, problems
from tests.conftest import cuda_available


def _sparse_m(A, seed):
    """diag(A)^-1 plus A's off-diagonal pattern with random values: a
    non-symmetric M with a realistic pattern."""
    rng = np.random.default_rng(seed)
    off = sparse.csc_matrix(A, copy=True)
    off.setdiag(0.0)
    off.eliminate_zeros()
    off.data = rng.uniform(-0.1, 0.1, off.nnz)
    return adjoint_oracle.canonical_csc(problems.diagonal_inverse(A) + off)


def _with_values(pattern, values):
    return sparse.csc_matrix((values, pattern.indices, pattern.indptr), shape=pattern.shape)


def _objective(A, M):
    return float(np.sum(adjoint_oracle.residual(A, M).data ** 2))


@pytest.mark.parametrize("maker", [lambda: problems.laplacian_2d(6), lambda: problems.diffusion_2d(5, 1.0, 2)])
def test_residual_adjoint_matches_finite_differences(maker):
    A = adjoint_oracle.canonical_csc(maker())
    M = _sparse_m(A, 3)
    loss, grad_m, grad_a = adjoint_oracle.residual_adjoint(A, M)
    assert loss == pytest.approx(_objective(A, M), rel=1e-13)
    rng = np.random.default_rng(4)
    for _ in range(6):
        dm = rng.standard_normal(M.nnz)
        da = rng.standard_normal(A.nnz)
        h = 1e-4
        # f is quadratic in M for fixed A (and in A for fixed M): central differences are exact up to rounding
        fd_m = (_objective(A, _with_values(M, M.data + h * dm)) - _objective(A, _with_values(M, M.data - h * dm))) / (2 * h)
        fd_a = (_objective(_with_values(A, A.data + h * da), M) - _objective(_with_values(A, A.data - h * da), M)) / (2 * h)
        assert grad_m @ dm == pytest.approx(fd_m, rel=1e-7, abs=1e-9)
        assert grad_a @ da == pytest.approx(fd_a, rel=1e-7, abs=1e-9)


def test_residual_adjoint_vanishes_at_the_exact_inverse():
    A = adjoint_oracle.canonical_csc(problems.tridiagonal(8).toarray())
    inverse = adjoint_oracle.canonical_csc(np.linalg.inv(A.toarray()))
    loss, grad_m, grad_a = adjoint_oracle.residual_adjoint(A, inverse)
    assert loss < 1e-28
    assert np.abs(grad_m).max() < 1e-13 and np.abs(grad_a).max() < 1e-13


def _symmetric_direction(A_csr, rng):
    """A random perturbation of A's stored values that keeps A symmetric."""
    upper = sparse.triu(A_csr, format="csr")
    upper.data = rng.standard_normal(upper.nnz)
    d = sparse.csr_matrix(upper + sparse.triu(upper, k=1).T)
    d.sort_indices()
    # d has A's pattern (A is symmetric), so its values line up with A.data
    assert np.array_equal(d.indices, A_csr.indices) and np.array_equal(d.indptr, A_csr.indptr)
    return d.data


def test_pcg_adjoint_math_matches_finite_differences():
    # L(A, b) = ||A^-1 b - x_t||^2 with a direct solve: checks dL/db = lambda, dL/dA = -lambda x^T
    A = sparse.csr_matrix(problems.diffusion_2d(8, 1.0, 7))
    A.sort_indices()
    rng = np.random.default_rng(8)
    x_t = rng.standard_normal(A.shape[0])
    b = A @ x_t + 0.01 * rng.standard_normal(A.shape[0])

    def loss(values, rhs):
        x = splinalg.spsolve(sparse.csc_matrix((values, A.indices, A.indptr), shape=A.shape).T.tocsc(), rhs)
        return float(np.sum((x - x_t) ** 2))

    x = splinalg.spsolve(A.tocsc(), b)
    lam = splinalg.spsolve(A.tocsc(), 2.0 * (x - x_t))
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    grad_a = -(lam[rows] * x[A.indices])
    for _ in range(8):
        da = _symmetric_direction(A, rng)
        db = rng.standard_normal(A.shape[0])
        h = 1e-6
        fd = (loss(A.data + h * da, b + h * db) - loss(A.data - h * da, b - h * db)) / (2 * h)
        assert grad_a @ da + lam @ db == pytest.approx(fd, rel=1e-6)


def test_pcg_adjoint_oracle_solves_the_adjoint_system():
    A = sparse.csr_matrix(problems.diffusion_2d(10, 1.0, 2))
    A.sort_indices()
    M = sparse.csr_matrix(problems.diagonal_inverse(A))
    rng = np.random.default_rng(1)
    x = rng.standard_normal(A.shape[0])
    g = rng.standard_normal(A.shape[0])
    lam, grad_a, history, status = adjoint_oracle.pcg_adjoint(A, M, x, g, 2000, 1e-12)
    assert status == 1 and history[-1] < 1e-12
    assert np.linalg.norm(A @ lam - g) <= 1e-10 * np.linalg.norm(g)
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    assert np.array_equal(grad_a, -(lam[rows] * x[A.indices]))


def _matrix_data(m):
    indptr = np.ascontiguousarray(m.indptr, np.int64)
    indices = np.ascontiguousarray(m.indices, np.int64)
    values = np.ascontiguousarray(m.data, np.float64)
    data = _lib.MatrixData(m.shape[0], m.shape[1], m.nnz, indptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                           indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                           values.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return data, (indptr, indices, values)


def test_residual_adjoint_rejects_bad_input_before_the_device():
    lib = _lib.load()
    A = adjoint_oracle.canonical_csc(problems.laplacian_2d(4))
    loss = ctypes.c_double(0.0)
    err = ctypes.create_string_buffer(256)

    def call(a, m):
        (ad, keep_a), (md, keep_m) = _matrix_data(a), _matrix_data(m)
        return lib.spai_residual_adjoint(ad, md, -1, ctypes.byref(loss), None, None, err, len(err))

    # rows out of order inside a column
    bad = A.copy()
    bad.indices[[0, 1]] = bad.indices[[1, 0]]
    assert call(A, bad) == -1 and b"strictly increasing" in err.value
    # size mismatch
    assert call(A, adjoint_oracle.canonical_csc(problems.laplacian_2d(3))) == -1
    assert b"same size" in err.value
    # the reference's own matrix checks come first (methods_c_api.cpp:16-40)
    empty = sparse.csc_matrix(A.shape)
    assert call(A, empty) == -1 and b"nnz must be positive" in err.value


def test_pcg_adjoint_rejects_bad_input_before_the_device():
    with pytest.raises(ValueError, match="same n"):
        adjoint.pcg_adjoint([1.0], [0], [0, 1], [1.0], [0], [0, 1], np.zeros(2), np.zeros(1), 10, 1e-8)
    lib = _lib.load()
    err = ctypes.create_string_buffer(256)
    params = _lib.PcgParams(10, 1e-8, 0, 0, -1, 0)
    one = np.ones(1)
    idx = np.zeros(1, np.int64)
    off = np.array([0, 1], np.int64)
    pf = ctypes.POINTER(ctypes.c_double)
    pi = ctypes.POINTER(ctypes.c_int64)
    count = lib.spai_pcg_adjoint(1, one.ctypes.data_as(pf), idx.ctypes.data_as(pi), off.ctypes.data_as(pi),
                                 one.ctypes.data_as(pf), idx.ctypes.data_as(pi), off.ctypes.data_as(pi), None, None,
                                 params, None, None, None, None, err, len(err))
    assert count == -1 and b"grad_x must not be null" in err.value


@pytest.mark.skipif(cuda_available(), reason="checks the no-device error path")
def test_adjoints_fail_loudly_without_a_device():
    A = problems.laplacian_2d(4)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        adjoint.residual_adjoint(A, problems.diagonal_inverse(A))
    Ac = sparse.csr_matrix(A)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        adjoint.pcg_adjoint(Ac.data, Ac.indices, Ac.indptr, Ac.data, Ac.indices, Ac.indptr, np.ones(16),
                            np.ones(16), 10, 1e-8)
