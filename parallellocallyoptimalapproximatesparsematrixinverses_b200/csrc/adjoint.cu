// Device adjoints of the SPAI objective and of the PCG solve (adjoint.cuh).
//
// The objective's gradient reuses the library's product kernels:
//   R      = I - A M        Spgemm, Epilogue::kResidual (per-column squares of
//                           R fused, reduced by the fixed tree into f);
//   dF/dM  = (A^T R)|M      SpgemmMasked with X = A^T, whose rows are A's
//                           columns, so A's own column-compressed copy serves;
//   dF/dA  = (R M^T)|A      SpgemmMasked with X = R (rows: the transpose of R)
//                           and B = M^T (columns: the transpose of M);
// then one pass scales both by -2 (exact in FP64).  All of it is memory-bound
// gather work of the same kind as the forward residual.

#include <cuda_runtime.h>

#include "adjoint.cuh"
#include "device.cuh"
#include "ops.cuh"
#include "spgemm.cuh"

namespace spai {

namespace {

__global__ void ScaleKernel(double* __restrict__ v, int64_t n, double s) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    v[i] = Mul(s, v[i]);
  }
}

// Warp per row i: lanes take the row's entries (coalesced), lambda_i is one
// broadcast load.
__global__ void NegativeOuterKernel(CscView<double> a_rows, const double* __restrict__ lambda,
                                    const double* __restrict__ x, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = warp; i < a_rows.cols; i += warps) {
    const double li = lambda[i];
    for (int64_t p = a_rows.ptr[i] + lane; p < a_rows.ptr[i + 1]; p += kWarp) {
      out[p] = -Mul(li, x[a_rows.idx[p]]);
    }
  }
}

void Scale(Ctx& ctx, double* v, int64_t n, double s) {
  if (n <= 0) return;
  ScaleKernel<<<GridFor(n, 256), 256, 0, ctx.stream>>>(v, n, s);
  SPAI_LAUNCH_CHECK();
}

}  // namespace

void ResidualAdjoint(Ctx& ctx, const DevCsc<double>& a, const DevCsc<double>& m, double* loss, double* grad_m,
                     double* grad_a) {
  const int64_t n = a.cols;
  DevCsc<double> a_rows;
  Transpose(ctx, a, a_rows);
  DevCsc<double> r;
  SpgemmExtras extras;
  extras.col_squares = ctx.Partial(0, n);
  Spgemm(ctx, a, a_rows, m, r, Epilogue::kResidual, extras);
  const double* parts[1] = {ctx.Partial(0, n)};
  TreeSums(ctx, parts, 1, n, 0);
  FetchScalars(ctx, 0, 1, loss);
  if (grad_m != nullptr && m.nnz > 0) {
    SpgemmMasked(ctx, a, r, m, grad_m);
    Scale(ctx, grad_m, m.nnz, -2.0);
  }
  if (grad_a != nullptr && a.nnz > 0) {
    DevCsc<double> r_rows;
    DevCsc<double> m_t;
    Transpose(ctx, r, r_rows);
    Transpose(ctx, m, m_t);
    SpgemmMasked(ctx, r_rows, m_t, a, grad_a);
    Scale(ctx, grad_a, a.nnz, -2.0);
  }
}

void NegativeOuterOnRows(Ctx& ctx, const DevCsc<double>& a_rows, const double* lambda, const double* x, double* out) {
  if (a_rows.nnz <= 0) return;
  NegativeOuterKernel<<<GridFor(a_rows.cols * kWarp, 256), 256, 0, ctx.stream>>>(View(a_rows), lambda, x, out);
  SPAI_LAUNCH_CHECK();
}

}  // namespace spai
