#pragma once
// Drop-in C ABI of the SPAI library, served by libspai_b200.so.
//
// Every struct below has the same field order, field types and size (8 bytes per
// field) as the reference's include/methods_c_api.h:7-46, and the five method
// entry points plus free_mem keep the reference's names and by-value signatures
// (include/methods_c_api.h:48-58), so code compiled against the reference header
// links against this library unchanged.  Like the reference header, the
// declarations sit inside `extern "C"` without a __cplusplus guard, so this
// header is meant for C++ translation units (C callers declare the same
// prototypes themselves, or use spai_b200.h which is C-clean).
//
// Semantics (reference src/common/methods_c_api.cpp:16-170):
//  * inputs are CSC, int64 col_offsets[cols+1] / row_indices[nnz], f64 values;
//    the pointers are borrowed and only read.  M0 and Pr are read only when
//    params.use_initial_m / params.use_preconditioner are non-zero.
//  * the returned arrays are allocated with new[] by the library; the caller
//    releases them with free_mem().  On failure every array is null and
//    error_message holds the text of the error.
//  * no exception crosses the ABI.

#include <stdint.h>

extern "C" {

// The same definitions appear in spai_b200.h; the guard lets both headers be
// included together.
#ifndef SPAI_ABI_STRUCTS_DEFINED
#define SPAI_ABI_STRUCTS_DEFINED
struct MatrixData {
  int64_t rows;
  int64_t cols;
  int64_t nnz;
  const int64_t* col_offsets;
  const int64_t* row_indices;
  const double* values;
};

struct MethodParams {
  int64_t max_iterations;
  double tolerance;
  double max_density;
  int64_t enable_dropping;
  int64_t num_threads;
  int64_t use_initial_m;
  int64_t use_preconditioner;
  int64_t inner_iterations;
};

struct SingleIterationData {
  int64_t iteration;
  double residual_norm;
  double density_m;
  double density_direction;
};

struct Result {
  int64_t rows;
  int64_t cols;
  int64_t nnz;
  int64_t iterations;
  int64_t converged;
  int64_t history_size;
  int64_t* col_offsets;
  int64_t* row_indices;
  double* values;
  SingleIterationData* history;
  char* error_message;
};
#endif  // SPAI_ABI_STRUCTS_DEFINED

// Global SPAI conjugate gradient   (reference src/global_spai/conjugate_gradient.cpp:15-83)
Result spai_global_cg(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params);

// Global SPAI minimal residual     (reference src/global_spai/minimal_residual.cpp:31-93)
Result spai_global_mr(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params);

// Global SPAI locally optimal MR   (reference src/global_spai/locally_minimal_residual.cpp:54-118)
Result spai_global_lomr(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params);

// Inner-Outer MR                   (reference src/inner_outer/inner_outer_common.hpp:14-107, locally_optimal=false)
Result inner_outer_mr(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params);

// Inner-Outer LOMR                 (reference src/inner_outer/inner_outer_common.hpp:14-107, locally_optimal=true)
Result inner_outer_lomr(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params);

// Releases the arrays of a Result and nulls them (reference src/common/methods_c_api.cpp:156-170).
void free_mem(Result* result);

}
