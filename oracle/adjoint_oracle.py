"""TEST INFRASTRUCTURE ONLY: CPU restatement of the device adjoints
(libspai_b200.so spai_residual_adjoint / spai_pcg_adjoint), used by tests/ as
the checker.  The reference has no adjoint; these follow the definitions:

  f(A, M) = ||I - A M||_F^2   (the squared residual norm of
                               methods_common.cpp:112-122)
  df/dM = -2 (A^T R) on M's pattern,  df/dA = -2 (R M^T) on A's pattern,
  R = I - A M;
  x = A^-1 b, upstream g = dL/dx:  A lambda = g,  dL/db = lambda,
  dL/dA(i, j) = -lambda_i x_j on A's pattern.

Arithmetic order, so that the device's FP64 results compare bit for bit:
scipy's CSR product sums each entry over k in the stored (ascending) order of
the left factor's row, first product first -- the device's masked product
order.  The loss is per-column sequential sums of squares in row order, then
the fixed 4096-wide tree (pyoracle.tree_sum).  lambda comes from the oracle
PCG in the device order.
"""
from __future__ import annotations

import numpy as np
from scipy import sparse

from . import pyoracle


def canonical_csc(matrix):
    m = sparse.csc_matrix(matrix, dtype=np.float64)
    m.sum_duplicates()
    m.sort_indices()
    return m


def residual(A, M):
    """R = I - A M as canonical CSC without stored zeros (dropping.cpp:97-104)."""
    A, M = canonical_csc(A), canonical_csc(M)
    R = sparse.csc_matrix(sparse.identity(A.shape[0], format="csc") - A @ M)
    R.eliminate_zeros()
    R.sort_indices()
    return R


def column_squares(X):
    """Per-column sum of squares, sequential in row order from +0.0."""
    X = canonical_csc(X)
    lengths = np.diff(X.indptr)
    sums = np.zeros(X.shape[1])
    squares = X.data * X.data
    for k in range(int(lengths.max(initial=0))):
        cols = np.nonzero(lengths > k)[0]
        sums[cols] = sums[cols] + squares[X.indptr[cols] + k]
    return sums


def _on_pattern(product, pattern):
    """Values of `product` at every stored entry of canonical CSC `pattern`."""
    product = sparse.csr_matrix(product)
    cols = np.repeat(np.arange(pattern.shape[1]), np.diff(pattern.indptr))
    return np.asarray(product[pattern.indices, cols]).ravel().astype(np.float64)


def residual_adjoint(A, M):
    """(f, grad on M's stored entries, grad on A's stored entries)."""
    A, M = canonical_csc(A), canonical_csc(M)
    R = residual(A, M)
    loss = pyoracle.tree_sum(column_squares(R))
    grad_m = -2.0 * _on_pattern(sparse.csr_matrix(A.T) @ sparse.csr_matrix(R), M)
    grad_a = -2.0 * _on_pattern(sparse.csr_matrix(R) @ sparse.csr_matrix(M.T), A)
    return loss, grad_m, grad_a


def pcg_adjoint(A, M, x, grad_x, max_iterations, tolerance, refresh_period=0):
    """(grad_b, grad on A's CSR entries, history, status) with lambda from the
    oracle PCG in the device order (A and M as CSR)."""
    A = sparse.csr_matrix(A, dtype=np.float64)
    A.sort_indices()
    history, status, lam = pyoracle.pcg(A, M, grad_x, max_iterations, tolerance, order=pyoracle.ORDER_DEVICE,
                                        refresh_period=refresh_period, return_x=True)
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    grad_a = -(lam[rows] * np.asarray(x, np.float64)[A.indices])
    return lam, grad_a, history, status
