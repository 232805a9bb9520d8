/* A plain C caller of the extended C ABI (include/spai_b200.h): it must
 * compile as C99 and link against libspai_b200.so.  Run on a GPU host it
 * builds M for tridiag(-1, 2, -1), n = 64, with Global MR and prints the last
 * residual; without a device the call returns the library's error text. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "spai_b200.h"

int main(void) {
  enum { n = 64 };
  int64_t offsets[n + 1];
  int64_t rows[3 * n];
  double values[3 * n];
  int64_t k = 0;
  for (int64_t j = 0; j < n; ++j) {
    offsets[j] = k;
    if (j > 0) { rows[k] = j - 1; values[k++] = -1.0; }
    rows[k] = j; values[k++] = 2.0;
    if (j + 1 < n) { rows[k] = j + 1; values[k++] = -1.0; }
  }
  offsets[n] = k;
  struct MatrixData a = {n, n, k, offsets, rows, values};
  struct MatrixData none = {0, 0, 0, NULL, NULL, NULL};
  struct MethodParams params = {10, 1e-12, 0.1, 1, 1, 0, 0, 2};
  SpaiExtParams ext = {0, 0, -1, 1};
  struct Result r = spai_run_ex(SPAI_GLOBAL_MR, a, none, none, params, &ext);
  if (r.error_message != NULL) {
    printf("error: %s\n", r.error_message);
    free_mem(&r);
    return 2;
  }
  printf("iterations %lld nnz %lld residual %.17g\n", (long long)r.iterations, (long long)r.nnz,
         r.history[r.history_size - 1].residual_norm);
  free_mem(&r);
  return 0;
}
