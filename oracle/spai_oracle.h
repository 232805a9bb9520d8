#pragma once
// TEST INFRASTRUCTURE ONLY.  CPU restatement ("oracle") of the reference's SPAI
// and PCG hot path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg may load the library built from this file; the product library
// (libspai_b200.so) never links or calls it.
//
// The oracle reproduces two summation orders for every global reduction:
//   order 0 "reference": per column-batch sequential sums in storage order,
//           then a sequential sum over batches (reference
//           src/common/methods_common.cpp:112-122 and every std::accumulate
//           over per-batch partials).  batch_count = min(n, num_threads) as in
//           the reference (methods_common.cpp:135-139).
//   order 1 "device": per column sequential sums in storage order, combined
//           by the fixed 4096-wide tree the CUDA library uses
//           (oracle_tree_sum below), so the CUDA results can be compared
//           bit for bit.
// Everything else (products, unions, pruning, selection) is order independent
// and identical in both modes.

#include <stdint.h>

#include "../include/methods_c_api.h"

extern "C" {

struct OracleOptions {
  int64_t order;            // 0 = reference batched order, 1 = device canonical order
  int64_t batch_count;      // order 0: column batches (0 -> params.num_threads); clamped to n
  int64_t omp_threads;      // OpenMP threads running the batches (0 -> batch count); results do not depend on it
  int64_t topk_per_column;  // 0 = reference global budget dropping; K>0 = keep at most K entries per column by magnitude
};

// method: 0 global CG, 1 global MR, 2 global LOMR, 3 inner-outer MR, 4 inner-outer LOMR.
// Same ownership rules as the C ABI: release with oracle_free.
Result oracle_run(int64_t method, MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params,
                  OracleOptions options);

void oracle_free(Result* result);

// PCG on CSR A and CSR M with x0 = 0 (reference methods_cython/backward_error.pyx:69-144).
// history must hold max_iterations doubles; returns the number written, *status gets 0..3.
// order 0 = sequential dot products (the reference with threads=1), 1 = device tree order.
// refresh_period > 0 additionally recomputes r = b - A x every refresh_period iterations.
int64_t oracle_pcg(int64_t n,
                   const double* a_values, const int64_t* a_indices, const int64_t* a_offsets,
                   const double* m_values, const int64_t* m_indices, const int64_t* m_offsets,
                   const double* b, int64_t max_iterations, double tolerance, int64_t order,
                   int64_t refresh_period, double* history, int64_t* status, double* x_out);

// The device's fixed summation tree over count values (exposed for tests).
double oracle_tree_sum(const double* values, int64_t count);

// Minimum-norm least-squares solve of a 2x2 system after symmetric diagonal
// scaling (reference src/common/sparse_operations.cpp:58-73).  Exposed for tests.
void oracle_solve_2x2(const double* matrix_row_major, const double* rhs, double* solution);

}
