// PCG evaluator on sm_100a.  Per iteration: two SpMVs (A p, M r), three dot
// products and the vector updates; all HBM-bound.  Dot products use the
// canonical tree of ops.cu over the elementwise products, so the CPU oracle
// reproduces every iterate bit for bit.

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "device.cuh"
#include "ops.cuh"
#include "pcg.cuh"
#include "profile.cuh"

namespace spai {

namespace {

// One thread per row, entries in storage order (the reference's _row_dot).
template <class TM>
__global__ void SpmvKernel(CscView<TM> a, const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t row = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; row < a.cols;
       row += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int64_t k = a.ptr[row]; k < a.ptr[row + 1]; ++k) {
      s = Add(s, Mul(static_cast<double>(a.val[k]), x[a.idx[k]]));
    }
    y[row] = s;
  }
}

// x += alpha p; r -= alpha Ap
__global__ void StepKernel(int64_t n, double alpha, const double* __restrict__ p, const double* __restrict__ ap,
                           double* __restrict__ x, double* __restrict__ r) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    x[i] = Add(x[i], Mul(alpha, p[i]));
    r[i] = __dsub_rn(r[i], Mul(alpha, ap[i]));
  }
}

// r = b - Ax
__global__ void TrueResidualKernel(int64_t n, const double* __restrict__ b, const double* __restrict__ ax,
                                   double* __restrict__ r) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    r[i] = __dsub_rn(b[i], ax[i]);
  }
}

// p = z + beta p
__global__ void DirectionKernel(int64_t n, double beta, const double* __restrict__ z, double* __restrict__ p) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    p[i] = Add(z[i], Mul(beta, p[i]));
  }
}

double DotProduct(Ctx& ctx, const double* x, const double* y, int64_t n) {
  const double* xs[1] = {x};
  const double* ys[1] = {y};
  TreeDots(ctx, xs, ys, 1, n, 0);
  double out;
  FetchScalars(ctx, 0, 1, &out);
  return out;
}

}  // namespace

template <class TM>
void Spmv(Ctx& ctx, const DevCsc<TM>& a_rows, const double* x, double* y) {
  // algorithmic bytes: the matrix once, x once, y written once
  const double bytes = static_cast<double>(a_rows.nnz) * (sizeof(TM) + sizeof(int32_t)) +
                       static_cast<double>(a_rows.cols + 1) * sizeof(int64_t) + 16.0 * static_cast<double>(a_rows.cols);
  prof::Scope scope(ctx.stream, "pcg_spmv", bytes);
  SpmvKernel<TM><<<GridFor(a_rows.cols, 128), 128, 0, ctx.stream>>>(View(a_rows), x, y);
  SPAI_LAUNCH_CHECK();
}

template <class TM>
void RunPcg(Ctx& ctx, const DevCsc<double>& a, const DevCsc<TM>& m, const double* b, double* x,
            const PcgOptions& opt, PcgResult& result) {
  const int64_t n = a.cols;
  DevBuf<double> r, z, p, ap;
  r.Reserve(static_cast<size_t>(n), ctx.stream);
  z.Reserve(static_cast<size_t>(n), ctx.stream);
  p.Reserve(static_cast<size_t>(n), ctx.stream);
  ap.Reserve(static_cast<size_t>(n), ctx.stream);
  const int grid = GridFor(n, 256);
  result.history.assign(1, 1.0);
  result.status = 0;
  result.spmv_count = 0;
  SPAI_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, ctx.stream));
  SPAI_CUDA(cudaMemcpyAsync(r.data(), b, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx.stream));
  Spmv(ctx, m, r.data(), z.data());
  ++result.spmv_count;
  SPAI_CUDA(cudaMemcpyAsync(p.data(), z.data(), sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx.stream));
  double r_r = DotProduct(ctx, r.data(), r.data(), n);
  const double b_norm = std::sqrt(r_r);
  double r_z = DotProduct(ctx, r.data(), z.data(), n);
  int64_t count = 1;
  int64_t status = 0;
  std::vector<double>& history = result.history;
  while (count < opt.max_iterations && history[count - 1] > opt.tolerance) {
    Spmv(ctx, a, p.data(), ap.data());
    ++result.spmv_count;
    const double den = DotProduct(ctx, p.data(), ap.data(), n);
    if (!std::isfinite(r_z) || !std::isfinite(den) || r_z == 0.0 || den == 0.0) {
      status = 2;
      break;
    }
    const double alpha = r_z / den;
    if (!std::isfinite(alpha)) {
      status = 2;
      break;
    }
    double beta = r_z;
    StepKernel<<<grid, 256, 0, ctx.stream>>>(n, alpha, p.data(), ap.data(), x, r.data());
    SPAI_LAUNCH_CHECK();
    r_r = DotProduct(ctx, r.data(), r.data(), n);
    double error = std::sqrt(r_r) / b_norm;
    const bool converged_refresh = error <= opt.tolerance;
    const bool periodic_refresh = opt.refresh_period > 0 && count % opt.refresh_period == 0;
    if (converged_refresh || periodic_refresh) {
      Spmv(ctx, a, x, ap.data());
      ++result.spmv_count;
      TrueResidualKernel<<<grid, 256, 0, ctx.stream>>>(n, b, ap.data(), r.data());
      SPAI_LAUNCH_CHECK();
      r_r = DotProduct(ctx, r.data(), r.data(), n);
      error = std::sqrt(r_r) / b_norm;
    }
    Spmv(ctx, m, r.data(), z.data());
    ++result.spmv_count;
    r_z = DotProduct(ctx, r.data(), z.data(), n);
    beta = converged_refresh ? 0.0 : r_z / beta;
    history.push_back(error);
    ++count;
    if (!std::isfinite(error)) {
      status = 3;
      break;
    }
    if (!std::isfinite(beta)) {
      status = 2;
      break;
    }
    DirectionKernel<<<grid, 256, 0, ctx.stream>>>(n, beta, z.data(), p.data());
    SPAI_LAUNCH_CHECK();
  }
  Spmv(ctx, a, x, ap.data());
  ++result.spmv_count;
  TrueResidualKernel<<<grid, 256, 0, ctx.stream>>>(n, b, ap.data(), r.data());
  SPAI_LAUNCH_CHECK();
  history[count - 1] = std::sqrt(DotProduct(ctx, r.data(), r.data(), n)) / b_norm;
  if (!std::isfinite(history[count - 1])) {
    status = 3;
  } else if (history[count - 1] <= opt.tolerance) {
    status = 1;
  }
  result.status = status;
  ctx.Sync();
}

template void RunPcg<double>(Ctx&, const DevCsc<double>&, const DevCsc<double>&, const double*, double*,
                             const PcgOptions&, PcgResult&);
template void RunPcg<float>(Ctx&, const DevCsc<double>&, const DevCsc<float>&, const double*, double*,
                            const PcgOptions&, PcgResult&);
template void Spmv<double>(Ctx&, const DevCsc<double>&, const double*, double*);
template void Spmv<float>(Ctx&, const DevCsc<float>&, const double*, double*);

}  // namespace spai
