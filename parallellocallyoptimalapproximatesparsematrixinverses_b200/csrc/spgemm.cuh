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
  // kResidual only: also write Z = diag(pr) * C with the same pattern into z_val.
  const void* row_scale = nullptr;  // T* pr
  void* z_val = nullptr;            // T* (capacity nnz(C)); pattern shared with C
  // kProjection: outputs
  double* proj_tt = nullptr;  // per column sum over rows of (pr_i c_i)^2
  double* proj_bt = nullptr;  // per column sum over rows in both of b_i * (pr_i c_i)
};

// x_csc and x_csr are the same matrix X in column and row compressed form.
// The C matrix (when written) replaces `c`.  `c_z` receives Z when
// extras.z_val is requested (same pattern, separate values).
template <class T>
void Spgemm(Ctx& ctx, const DevCsc<T>& x_csc, const DevCsc<T>& x_csr, const DevCsc<T>& b, DevCsc<T>& c,
            Epilogue epilogue, SpgemmExtras extras = SpgemmExtras(), DevCsc<T>* c_z = nullptr);

// Masked product: out[p] = (X*B)(row(p), col(p)) for every entry p of the
// pattern matrix `mask` (0.0 where the product has no term), values in FP64.
template <class T>
void SpgemmMasked(Ctx& ctx, const DevCsc<T>& x_csr, const DevCsc<T>& b, const DevCsc<T>& mask, double* out);

}  // namespace spai
