#pragma once
// Preconditioned conjugate gradients with a sparse approximate inverse M
// (reference methods_cython/backward_error.pyx:69-144).  A and M are held as
// row-compressed matrices in HBM (DevCsc with rows as the major dimension);
// M may be stored in FP32 (mixed precision) while every vector, dot product
// and the true-residual refresh stay in FP64.

#include <cstdint>
#include <vector>

#include "device.cuh"
#include "ops.cuh"

namespace spai {

struct PcgOptions {
  int64_t max_iterations = 50;  // history length limit, includes the initial entry
  double tolerance = 1e-6;
  int64_t refresh_period = 0;   // > 0: also replace r by b - A x every refresh_period iterations
};

struct PcgResult {
  std::vector<double> history;
  int64_t status = 0;  // 0 iteration limit, 1 converged, 2 recurrence breakdown, 3 non-finite residual
  int64_t spmv_count = 0;
};

// Solves with x0 = 0; b and x are device vectors of length a.rows.
template <class TM>
void RunPcg(Ctx& ctx, const DevCsc<double>& a_rows, const DevCsc<TM>& m_rows, const double* b, double* x,
            const PcgOptions& options, PcgResult& result);

// y = A x for a row-compressed A (reference backward_error.pyx:27-34, per row sequential).
template <class TM>
void Spmv(Ctx& ctx, const DevCsc<TM>& a_rows, const double* x, double* y);

}  // namespace spai
