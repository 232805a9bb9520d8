#pragma once
// Two-phase SpGEMM C = X * B on column-compressed matrices (the reference's
// Eigen sparse product, state_manager.cpp:59, dropping.cpp:98,
// inner_outer_common.hpp:48).
//
// Phase 1 (symbolic) counts the distinct rows of every output column with a
// shared-memory hash; phase 2 (numeric) rebuilds the row set, sorts it, and
// computes every output entry by pulling row i of X (CSR copy) against a
// hash of column j of B.  The pull visits k in ascending order, so each entry
// is the first product x*y followed by += x*y in ascending k -- exactly the
// reference's accumulation order, with no FMA.

#include "device.cuh"
#include "ops.cuh"

namespace spai {

enum class Epilogue {
  kPlain = 0,       // C = X*B, structural zeros kept (dropping enabled in the reference)
  kPruneZeros = 1,  // C = X*B, exact zeros removed (dropping disabled)
  kResidual = 2,    // C = I - X*B with the diagonal inserted, exact zeros removed
  kProjection = 3,  // no output: per column sum((pr*c)^2) and sum(b*(pr*c)) (fused MR projection)
};

struct SpgemmExtras {
  // Optional per-column partial sum of squares of the output column (storage order).
  double* col_squares = nullptr;
  // kResidual: Z = diag(row_scale) * C is also written when c_z is given;
  // kProjection: the row scale pr.
  const void* row_scale = nullptr;  // const T*
  // kProjection: outputs
  double* proj_tt = nullptr;  // per column sum over rows of (pr_i c_i)^2
  double* proj_bt = nullptr;  // per column sum over rows in both of b_i * (pr_i c_i)
  // Optional fixed-width (ELL) copies of X with `ell_width` slots per column /
  // row (a multiple of 4), entries in storage order, padded with index -1:
  // the column kernel then reads a whole column or row of X with 16-byte loads.
  const int32_t* x_cols_ell = nullptr;      // rows of X(:, k)
  const int32_t* x_rows_ell = nullptr;      // columns of X(i, :)
  const void* x_rows_ell_val = nullptr;     // values of X(i, :) (const T*)
  int ell_width = 0;
};

// x_csc and x_csr are the same matrix X in column and row compressed form.
// The C matrix (when written) replaces `c`.  For kResidual with
// extras.row_scale set and c_z given, Z = diag(row_scale) * C is written into
// c_z as well; the return value says whether it was (it is not when an exact
// zero had to be pruned from C).
template <class T>
bool Spgemm(Ctx& ctx, const DevCsc<T>& x_csc, const DevCsc<T>& x_csr, const DevCsc<T>& b, DevCsc<T>& c,
            Epilogue epilogue, SpgemmExtras extras = SpgemmExtras(), DevCsc<T>* c_z = nullptr);

// Masked product: out[p] = (X*B)(row(p), col(p)) for every entry p of the
// pattern matrix `mask` (0.0 where the product has no term), values in FP64.
template <class T>
void SpgemmMasked(Ctx& ctx, const DevCsc<T>& x_csr, const DevCsc<T>& b, const DevCsc<T>& mask, double* out);

}  // namespace spai
