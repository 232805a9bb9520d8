#pragma once
// The fused, graph-captured Global MR iteration (reference
// src/global_spai/minimal_residual.cpp:55-89) for the per-column top-k drop
// with a diagonal Pr and a stencil-like A (ELL copies of at most 16 entries
// per row and column), in the device summation order.
//
// One iteration is three kernels:
//   drop      M := top-k(threshold(0.5 (U + U^T))) with U = M + alpha Z formed
//             on the fly: column j from M's and Z's slots, row j from M^T and
//             row j of A (row j of Z is recomputed, never transposed); writes
//             M in place and scatters M^T;
//   residual  R = I - A M, Z = Pr R written, the column squares of R, and the
//             MR projection of A Z from the Z column still in shared memory
//             (no second pass over Z);
//   decide    the three fixed-tree reductions (||R||^2, <Z, Pr A Z>,
//             ||Pr A Z||^2), the history row, the stop tests and the next
//             step length, all on the device; it sets the condition of the
//             CUDA graph's WHILE node that repeats the three kernels.
// Matrices live in fixed-capacity column slots (M: topk per column; Z: the
// bound 1 + topk * (longest column of A); M^T: per-row slots), so no
// size is read back and no allocation happens inside the loop.  Every value
// is formed with the same operations, in the same order, as the unfused
// kernels (update.cu, spgemm.cu), so results are bit-identical.  A column
// that does not fit its slots flags an overflow: the loop stops and the
// caller reruns the solve on the unfused path.

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "device.cuh"
#include "ops.cuh"
#include "solver.cuh"

namespace spai {

struct FusedMrProblem {
  int64_t n = 0;
  int topk = 0;
  int64_t a_nnz = 0;
  int64_t a_longest = 0;                 // longest column (or row) of A
  int ell_width = 0;                     // slots of the ELL copies of A
  const int32_t* a_cols_ell = nullptr;   // rows of A(:, k)
  const int32_t* a_rows_ell = nullptr;   // columns of A(i, :)
  const void* a_rows_ell_val = nullptr;  // values of A(i, :) (T)
  const void* pr = nullptr;              // diag(Pr) (T)
  int64_t max_iterations = 0;
  double tolerance = 0.0;
};

// Outcome of a fused run.
struct FusedMrOutcome {
  bool ran = false;        // false: the fused loop did not apply (nothing changed)
  bool overflow = false;   // a column did not fit: the caller reruns on the unfused path
  bool converged = false;
  int64_t iterations = 0;  // the last history row appended
  int64_t graph_bodies = 0;
};

class FusedMrBase {
 public:
  virtual ~FusedMrBase() = default;
  // Continues Global MR from the state after iteration 0: m and z (Z = Pr R)
  // as compact CSC (DevCsc<T>), the first step length alpha.  Appends rows
  // 1.. to `history` and replaces m with the final M.
  virtual FusedMrOutcome Run(Ctx& ctx, const FusedMrProblem& problem, void* m_csc, const void* z_csc, double alpha,
                             std::vector<SingleIterationData>& history) = 0;
};

// Whether the fused loop can take the problem (slot and window capacities).
bool FusedMrApplicable(const FusedMrProblem& problem);

// Process-wide switch (spai_set_fused_mr): off, every Global MR runs on the
// unfused kernels, which give the same bits; tests compare the two.
bool FusedMrEnabled();
void SetFusedMrEnabled(bool enabled);

template <class T>
std::unique_ptr<FusedMrBase> MakeFusedMr();

}  // namespace spai
