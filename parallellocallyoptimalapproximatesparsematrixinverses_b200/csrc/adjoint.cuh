#pragma once
// Reverse mode (adjoints) of the SPAI objective and of the PCG solve.  The
// reference computes neither; they differentiate the quantities it does
// compute, so a caller can fit A's values or M's values by gradient descent.
//
// Objective f(A, M) = ||I - A M||_F^2, the square of the residual norm the
// reference records every iteration (methods_common.cpp:112-122):
//   df/dM(i, j) = -2 (A^T R)(i, j)  at every stored entry (i, j) of M,
//   df/dA(i, k) = -2 (R M^T)(i, k)  at every stored entry (i, k) of A,
// with R = I - A M.  Both are masked products: one thread per stored entry
// sums its terms in ascending k, the order of every other product here.
//
// PCG solve x = A^-1 b (backward_error.pyx:69-144) with an upstream gradient
// g = dL/dx: the implicit-function adjoint solves A^T lambda = g -- A is
// symmetric, so this is a second PCG with the forward's preconditioner -- and
//   dL/db = lambda,   dL/dA(i, j) = -lambda_i x_j  at every stored entry.
// The gradient is that of the exact solution map A^-1 b; it matches the
// gradient of the computed x to the solve's tolerance, and needs no stored
// iterates (O(n) memory, independent of the iteration count).

#include "device.cuh"
#include "ops.cuh"

namespace spai {

// a and m column-compressed FP64 (n x n).  *loss = f (per-column sums in row
// order, then the fixed 4096-wide tree); grad_m (nnz(m)) and grad_a (nnz(a))
// are device arrays in the matrices' storage order, either may be null.
void ResidualAdjoint(Ctx& ctx, const DevCsc<double>& a, const DevCsc<double>& m, double* loss, double* grad_m,
                     double* grad_a);

// out[q] = -(lambda_i * x_j) at every entry q = (i, j) of the row-compressed
// matrix a_rows (device arrays).
void NegativeOuterOnRows(Ctx& ctx, const DevCsc<double>& a_rows, const double* lambda, const double* x, double* out);

}  // namespace spai
