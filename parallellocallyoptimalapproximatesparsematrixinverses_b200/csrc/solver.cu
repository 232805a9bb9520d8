// Device implementation of Global SPAI CG / MR / LOMR and Inner-Outer MR /
// LOMR.  Each method follows the reference's control flow line for line
// (file:line given at each method); the arithmetic of every step runs in the
// kernels of ops.cu and spgemm.cu.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <thread>
#include <type_traits>
#include <vector>

#include "cod2x2.cuh"
#include "device.cuh"
#include "mr_fused.cuh"
#include "ops.cuh"
#include "solver.cuh"
#include "spgemm.cuh"

namespace spai {

namespace {

constexpr double kEpsilon = std::numeric_limits<double>::epsilon();  // methods_common.hpp:32
constexpr double kMinDensity = 1e-9;                                 // include/methods.hpp:15

__device__ __forceinline__ bool FiniteNonZero(double v) { return isfinite(v) && fabs(v) > 0.0; }

__device__ __forceinline__ double SafeQuotient(double num, double den) {
  if (!FiniteNonZero(den)) return 0.0;
  const double q = __ddiv_rn(num, den);
  return isfinite(q) ? q : 0.0;
}

// The reference's summation order: thread per column batch, sequential over
// the batch's columns in storage order (AccSquares / AccDot of a batch).
template <class T>
__global__ void BatchSquaresKernel(CscView<T> x, const int64_t* __restrict__ first, int64_t batches,
                                   double* __restrict__ out) {
  for (int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < batches;
       b += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int64_t p = x.ptr[first[b]]; p < x.ptr[first[b + 1]]; ++p) {
      const double v = static_cast<double>(x.val[p]);
      s = Add(s, Mul(v, v));
    }
    out[b] = s;
  }
}

template <class T>
__global__ void BatchDotsKernel(CscView<T> x, CscView<T> y, const int64_t* __restrict__ first, int64_t batches,
                                double* __restrict__ out) {
  for (int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < batches;
       b += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int64_t j = first[b]; j < first[b + 1]; ++j) {
      int64_t p = x.ptr[j];
      int64_t q = y.ptr[j];
      const int64_t pe = x.ptr[j + 1];
      const int64_t qe = y.ptr[j + 1];
      while (p < pe && q < qe) {
        const int32_t rp = x.idx[p];
        const int32_t rq = y.idx[q];
        if (rp == rq) {
          s = Add(s, Mul(static_cast<double>(x.val[p]), static_cast<double>(y.val[q])));
          ++p;
          ++q;
        } else if (rp < rq) {
          ++p;
        } else {
          ++q;
        }
      }
    }
    out[b] = s;
  }
}

// Canonical device CSC (int64 offsets and rows) -> int32 rows in dst, with
// *bad |= 1 for offsets that do not run from 0 to nnz or decrease, and
// |= 2 for rows out of [0, n) or not strictly increasing in a column.
__global__ void CheckNarrowCscKernel(int64_t n, int64_t nnz, const int64_t* __restrict__ ptr,
                                     const int64_t* __restrict__ idx, int32_t* __restrict__ dst,
                                     int32_t* __restrict__ bad) {
  int flags = 0;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = ptr[j];
    const int64_t e = ptr[j + 1];
    if ((j == 0 && b != 0) || (j == n - 1 && e != nnz) || e < b || b < 0 || e > nnz) {
      flags |= 1;
      continue;
    }
    int64_t previous = -1;
    for (int64_t p = b; p < e; ++p) {
      const int64_t r = idx[p];
      if (r < 0 || r >= n || r <= previous) flags |= 2;
      previous = r;
      dst[p] = static_cast<int32_t>(r);
    }
  }
  if (flags != 0) atomicOr(bad, flags);
}

// The longest column of x and the longest row (the longest column of its
// transpose) into out[0] (out zeroed by the caller).
__global__ void LongestKernel(const int64_t* __restrict__ ptr_a, const int64_t* __restrict__ ptr_b, int64_t n,
                              unsigned long long* __restrict__ out) {
  unsigned long long m = 0;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned long long a = static_cast<unsigned long long>(ptr_a[j + 1] - ptr_a[j]);
    const unsigned long long b = static_cast<unsigned long long>(ptr_b[j + 1] - ptr_b[j]);
    m = a > m ? a : m;
    m = b > m ? b : m;
  }
  if (m != 0ull) atomicMax(out, m);
}

// pr[j] = 1 / A(j, j) (methods_common.cpp:50-63); *bad |= 1 for a missing,
// non-positive or non-finite diagonal, |= 2 for a non-finite inverse.
template <class T>
__global__ void DiagonalInverseKernel(CscView<double> a, T* __restrict__ pr, int32_t* __restrict__ bad) {
  int flags = 0;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < a.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t lo = a.ptr[j];
    int64_t hi = a.ptr[j + 1];
    while (lo < hi) {
      const int64_t mid = lo + ((hi - lo) >> 1);
      if (a.idx[mid] < j) {
        lo = mid + 1;
      } else {
        hi = mid;
      }
    }
    const double d = (lo < a.ptr[j + 1] && a.idx[lo] == j) ? a.val[lo] : 0.0;
    if (!isfinite(d) || d <= 0.0) {
      flags |= 1;
      continue;
    }
    const double inverse = __ddiv_rn(1.0, d);
    if (!isfinite(inverse)) flags |= 2;
    pr[j] = static_cast<T>(inverse);
  }
  if (flags != 0) atomicOr(bad, flags);
}

// int32 rows and T values -> int64 and FP64 (device to device).
template <class T>
__global__ void WidenKernel(const int32_t* __restrict__ idx, const T* __restrict__ val, int64_t n,
                            int64_t* __restrict__ idx_out, double* __restrict__ val_out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    idx_out[i] = static_cast<int64_t>(idx[i]);
    val_out[i] = static_cast<double>(val[i]);
  }
}

// out[i] = ptr[at[i]]: the column offsets of a matrix at the block boundaries.
__global__ void GatherOffsetsKernel(const int64_t* __restrict__ ptr, const int64_t* __restrict__ at, int64_t count,
                                    int64_t* __restrict__ out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[i] = ptr[at[i]];
  }
}

// per_column[j] = per_block[block of column j].
__global__ void BroadcastBlocksKernel(const int32_t* __restrict__ block_of, const double* __restrict__ per_block,
                                      int64_t n, double* __restrict__ per_column) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    per_column[j] = per_block[block_of[j]];
  }
}

// Per-column Inner-Outer step lengths (inner_outer_common.hpp:50-69).
__global__ void InnerOuterStepKernel(int64_t n, const double* __restrict__ r_az, const double* __restrict__ az_az,
                                     const double* __restrict__ az_aq, const double* __restrict__ aq_aq,
                                     const double* __restrict__ r_aq, bool locally_optimal, bool first,
                                     double* __restrict__ delta, double* __restrict__ gamma,
                                     double* __restrict__ normalization) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double d;
    double g;
    if (!locally_optimal || first) {
      d = SafeQuotient(r_az[j], az_az[j]);
      g = locally_optimal ? 1.0 : 0.0;
    } else {
      const double gram[4] = {az_az[j], az_aq[j], az_aq[j], aq_aq[j]};
      const double rhs[2] = {r_az[j], r_aq[j]};
      double coef[2];
      SolveLeastSquares2x2(gram, rhs, coef);
      d = coef[0];
      g = coef[1];
    }
    delta[j] = d;
    gamma[j] = g;
    const double inverse = d != 0.0 ? __ddiv_rn(1.0, d) : 1.0;
    normalization[j] = isfinite(inverse) ? inverse : 1.0;
  }
}

__global__ void SafeQuotientKernel(int64_t n, const double* __restrict__ num, const double* __restrict__ den,
                                   double* __restrict__ out) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[j] = SafeQuotient(num[j], den[j]);
  }
}

__global__ void IdentityKernel(int64_t n, int64_t* __restrict__ ptr, int32_t* __restrict__ idx) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j <= n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    ptr[j] = j;
    if (j < n) idx[j] = static_cast<int32_t>(j);
  }
}

template <class T>
__global__ void FillKernel(T* __restrict__ out, int64_t n, T value) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[i] = value;
  }
}

__global__ void NarrowIndexKernel(const int64_t* __restrict__ src, int32_t* __restrict__ dst, int64_t n) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    dst[i] = static_cast<int32_t>(src[i]);
  }
}

}  // namespace

// A canonical CSC in device memory -> out (int32 rows), checked on the device.
void UploadCheckedDeviceCsc(Ctx& ctx, const DeviceCscInput& in, DevCsc<double>& out, const char* name) {
  out.Shape(in.n, in.n, ctx.stream);
  out.ReserveNnz(in.nnz, ctx.stream);
  SPAI_CUDA(cudaMemcpyAsync(out.ptr.data(), in.col_offsets, sizeof(int64_t) * (in.n + 1), cudaMemcpyDeviceToDevice,
                            ctx.stream));
  if (in.nnz > 0) {
    SPAI_CUDA(cudaMemcpyAsync(out.val.data(), in.values, sizeof(double) * in.nnz, cudaMemcpyDeviceToDevice,
                              ctx.stream));
  }
  int32_t* bad = ctx.flags.data() + 5;
  SPAI_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), ctx.stream));
  CheckNarrowCscKernel<<<GridFor(in.n, 128), 128, 0, ctx.stream>>>(in.n, in.nnz, in.col_offsets, in.row_indices,
                                                                   out.idx.data(), bad);
  SPAI_LAUNCH_CHECK();
  SPAI_CUDA(cudaMemcpyAsync(ctx.host_flags + 5, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();
  if (ctx.host_flags[5] & 1) {
    throw std::invalid_argument(std::string(name) + ": column offsets must run from 0 to nnz without decreasing");
  }
  if (ctx.host_flags[5] & 2) {
    throw std::invalid_argument(std::string(name) +
                                ": row indices must lie in [0, n) and increase strictly in every column");
  }
}

template <class T>
void UploadCsc(Ctx& ctx, const HostCsc& h, DevCsc<T>& d, DevBuf<int64_t>& stage_idx, DevBuf<double>& stage_val) {
  d.Shape(h.rows, h.cols, ctx.stream);
  // column offsets are rebased so the device matrix starts at 0
  std::vector<int64_t> ptr(h.cols + 1);
  const int64_t base = h.ptr[0];
  for (int64_t j = 0; j <= h.cols; ++j) ptr[j] = h.ptr[j] - base;
  const int64_t nnz = ptr[h.cols];
  d.ReserveNnz(nnz, ctx.stream);
  SPAI_CUDA(cudaMemcpyAsync(d.ptr.data(), ptr.data(), sizeof(int64_t) * (h.cols + 1), cudaMemcpyHostToDevice,
                            ctx.stream));
  if (nnz > 0) {
    stage_idx.Reserve(static_cast<size_t>(nnz), ctx.stream);
    SPAI_CUDA(cudaMemcpyAsync(stage_idx.data(), h.idx + base, sizeof(int64_t) * nnz, cudaMemcpyHostToDevice,
                              ctx.stream));
    NarrowIndexKernel<<<GridFor(nnz, 256), 256, 0, ctx.stream>>>(stage_idx.data(), d.idx.data(), nnz);
    SPAI_LAUNCH_CHECK();
    if (std::is_same<T, double>::value) {
      SPAI_CUDA(cudaMemcpyAsync(d.val.data(), h.val + base, sizeof(double) * nnz, cudaMemcpyHostToDevice,
                                ctx.stream));
    } else {
      stage_val.Reserve(static_cast<size_t>(nnz), ctx.stream);
      SPAI_CUDA(cudaMemcpyAsync(stage_val.data(), h.val + base, sizeof(double) * nnz, cudaMemcpyHostToDevice,
                                ctx.stream));
      ConvertValues<double, T>(ctx, stage_val.data(), d.val.data(), nnz);
    }
  }
  // the pageable host arrays must stay valid until the copies finish
  ctx.Sync();
}

template void UploadCsc<double>(Ctx&, const HostCsc&, DevCsc<double>&, DevBuf<int64_t>&, DevBuf<double>&);
template void UploadCsc<float>(Ctx&, const HostCsc&, DevCsc<float>&, DevBuf<int64_t>&, DevBuf<double>&);

namespace {

template <class T>
class Solver final : public SolverBase {
 public:
  Solver(Ctx& ctx, const SolveOptions& options) : ctx_(ctx), opt_(options) {}

  void Upload(const HostCsc& a, const HostCsc* m0, const HostCsc* pr) override {
    n_ = a.cols;
    DevBuf<int64_t> stage_idx;
    DevBuf<double> stage_val;
    UploadCsc(ctx_, a, a64_, stage_idx, stage_val);
    SetUpFromA();
    // preconditioner (methods_common.cpp:105-110)
    pr_diagonal_ = true;
    if (pr != nullptr) {
      pr_diagonal_ = IsFullDiagonal(*pr);
      if (pr_diagonal_) {
        std::vector<T> host(n_);
        for (int64_t j = 0; j < n_; ++j) host[j] = static_cast<T>(pr->val[pr->ptr[j]]);
        pr_vec_.Reserve(static_cast<size_t>(n_), ctx_.stream);
        SPAI_CUDA(cudaMemcpyAsync(pr_vec_.data(), host.data(), sizeof(T) * n_, cudaMemcpyHostToDevice, ctx_.stream));
        ctx_.Sync();
      } else {
        UploadCsc(ctx_, *pr, pr_, stage_idx, stage_val);
        Transpose(ctx_, pr_, pr_csr_);
      }
    } else {
      DiagonalInversePreconditioner();
    }
    // M0 (methods_common.cpp:78-103): given, or the identity
    if (m0 != nullptr) {
      UploadCsc(ctx_, *m0, m0_, stage_idx, stage_val);
    } else {
      IdentityM0();
    }
    ctx_.Sync();
  }

  void UploadDevice(const DeviceCscInput& a, const DeviceCscInput* m0) override {
    n_ = a.n;
    CopyCheckedFromDevice(a, a64_, "A");
    SetUpFromA();
    pr_diagonal_ = true;
    DiagonalInversePreconditioner();
    if (m0 != nullptr) {
      DevCsc<double> m64;
      CopyCheckedFromDevice(*m0, m64, "M0");
      if constexpr (std::is_same<T, double>::value) {
        m0_.Swap(m64);
      } else {
        ConvertCsc(m64, m0_);
      }
    } else {
      IdentityM0();
    }
    ctx_.Sync();
  }

  void Run() override {
    RunOnce();
    if (fused_overflowed_) {
      // a column outgrew the fused loop's slots: the same solve on the unfused kernels (same bits)
      fused_allowed_ = false;
      RunOnce();
    }
  }

  void RunOnce() {
    fused_overflowed_ = false;
    history_.clear();
    converged_ = false;
    iterations_ = 0;
    Copy(ctx_, m0_, m_);
    for (DevCsc<T>* x : {&r_, &z_, &p_, &ap_, &az_, &tmp_, &q_}) Empty(*x);
    InvalidateResidualExtras();
    const bool inner_outer = opt_.method == Method::kInnerOuterMr || opt_.method == Method::kInnerOuterLomr;
    symmetric_ = !inner_outer;
    // PrepareStateManager (methods_common.cpp:126-157)
    if (opt_.dropping) {
      ApplyDroppingStrategy();
    } else {
      Residual();
    }
    initial_residual_ = std::sqrt(SquaredNorm(r_));
    switch (opt_.method) {
      case Method::kGlobalCg: RunCg(); break;
      case Method::kGlobalMr: RunMr(); break;
      case Method::kGlobalLomr: RunLomr(); break;
      case Method::kInnerOuterMr: RunInnerOuter(false); break;
      case Method::kInnerOuterLomr: RunInnerOuter(true); break;
    }
    ctx_.Sync();
  }

  void Download(SolveOutput& out) override {
    out.Allocate(m_.rows, m_.cols, m_.nnz);
    DownloadM(out.ptr.get(), out.idx.get(), out.val.get());
    out.history = history_;
    out.iterations = iterations_;
    out.converged = converged_;
  }

  void DownloadM(int64_t* ptr, int64_t* idx, double* val) override {
    SPAI_CUDA(cudaMemcpyAsync(ptr, m_.ptr.data(), sizeof(int64_t) * (m_.cols + 1), cudaMemcpyDeviceToHost,
                              ctx_.stream));
    DownloadWiden<T>(ctx_, m_.idx.data(), m_.val.data(), m_.nnz, 0, idx, val);
    ctx_.Sync();
  }

  void ExportMDevice(int64_t* ptr, int64_t* idx, double* val) override {
    SPAI_CUDA(cudaMemcpyAsync(ptr, m_.ptr.data(), sizeof(int64_t) * (m_.cols + 1), cudaMemcpyDeviceToDevice,
                              ctx_.stream));
    if (m_.nnz > 0) {
      WidenKernel<T><<<GridFor(m_.nnz, 256), 256, 0, ctx_.stream>>>(m_.idx.data(), m_.val.data(), m_.nnz, idx, val);
      SPAI_LAUNCH_CHECK();
    }
    ctx_.Sync();
  }

  const std::vector<SingleIterationData>& history() const override { return history_; }
  bool converged() const override { return converged_; }

  // Batched Global MR: the loop of RunMr (minimal_residual.cpp:31-93) per
  // diagonal block.  Every block follows the single-system arithmetic bit for
  // bit: the products, unions and drop steps are column-local, and each
  // block's scalars come from the fixed tree over that block's columns
  // (SegmentTree).  A block that stops (converged, density limit, breakdown,
  // iteration limit) has its M copied out at that moment; afterwards it rides
  // along with step length 0 and its results are no longer read.
  void RunMrBatched(const std::vector<int64_t>& offsets, std::vector<SolveOutput>& outputs) override {
    const int64_t blocks = static_cast<int64_t>(offsets.size()) - 1;
    if (blocks <= 0 || offsets.front() != 0 || offsets.back() != n_) throw std::invalid_argument("bad block offsets");
    if (!pr_diagonal_) throw std::invalid_argument("batched runs use a diagonal Pr");
    if (opt_.dropping && opt_.topk <= 0) throw std::invalid_argument("batched runs need top-k dropping or none");
    SegmentTree tree;
    tree.Build(ctx_, offsets);
    std::vector<int32_t> block_of(static_cast<size_t>(n_));
    for (int64_t b = 0; b < blocks; ++b) {
      for (int64_t j = offsets[b]; j < offsets[b + 1]; ++j) block_of[j] = static_cast<int32_t>(b);
    }
    DevBuf<int32_t> block_of_dev;
    DevBuf<int64_t> bounds_dev;
    DevBuf<int64_t> gathered;
    DevBuf<double> alpha_dev;
    block_of_dev.Reserve(static_cast<size_t>(n_), ctx_.stream);
    bounds_dev.Reserve(static_cast<size_t>(blocks + 1), ctx_.stream);
    gathered.Reserve(static_cast<size_t>(2 * (blocks + 1)), ctx_.stream);
    alpha_dev.Reserve(static_cast<size_t>(blocks), ctx_.stream);
    SPAI_CUDA(cudaMemcpyAsync(block_of_dev.data(), block_of.data(), sizeof(int32_t) * n_, cudaMemcpyHostToDevice,
                              ctx_.stream));
    SPAI_CUDA(cudaMemcpyAsync(bounds_dev.data(), offsets.data(), sizeof(int64_t) * (blocks + 1),
                              cudaMemcpyHostToDevice, ctx_.stream));
    ctx_.Sync();

    outputs.clear();
    outputs.resize(static_cast<size_t>(blocks));
    std::vector<char> active(static_cast<size_t>(blocks), 1);
    int64_t live = blocks;
    std::vector<double> sums(static_cast<size_t>(2 * blocks));
    std::vector<int64_t> m_at(static_cast<size_t>(blocks + 1));
    std::vector<int64_t> z_at(static_cast<size_t>(blocks + 1));
    std::vector<int> stopping;

    // nnz of M and Z per block: their column offsets at the block boundaries
    auto fetch_counts = [&]() {
      const int g = GridFor(blocks + 1, 128);
      GatherOffsetsKernel<<<g, 128, 0, ctx_.stream>>>(m_.ptr.data(), bounds_dev.data(), blocks + 1, gathered.data());
      SPAI_LAUNCH_CHECK();
      GatherOffsetsKernel<<<g, 128, 0, ctx_.stream>>>(z_.ptr.data(), bounds_dev.data(), blocks + 1,
                                                      gathered.data() + blocks + 1);
      SPAI_LAUNCH_CHECK();
      SPAI_CUDA(cudaMemcpyAsync(m_at.data(), gathered.data(), sizeof(int64_t) * (blocks + 1), cudaMemcpyDeviceToHost,
                                ctx_.stream));
      SPAI_CUDA(cudaMemcpyAsync(z_at.data(), gathered.data() + blocks + 1, sizeof(int64_t) * (blocks + 1),
                                cudaMemcpyDeviceToHost, ctx_.stream));
      ctx_.Sync();
    };
    // ||R||_F per block from the column squares the last residual product left
    auto residual_norms = [&](std::vector<double>& out) {
      if (!r_squares_ready_) ColumnSquares(ctx_, View(r_), ctx_.Partial(kResidualPartial, n_));
      const double* parts[1] = {ctx_.Partial(kResidualPartial, n_)};
      tree.Sums(ctx_, parts, 1, sums.data());
      out.resize(static_cast<size_t>(blocks));
      for (int64_t b = 0; b < blocks; ++b) out[b] = std::sqrt(sums[b]);
    };
    // M of every block in `stopping` to its output (local indices, FP64 values)
    auto snapshot = [&]() {
      if (stopping.empty()) return;
      fetch_counts();
      for (const int b : stopping) {
        SolveOutput& out = outputs[b];
        const int64_t c0 = offsets[b];
        const int64_t cols = offsets[b + 1] - c0;
        const int64_t p0 = m_at[b];
        const int64_t nnz = m_at[b + 1] - p0;
        out.Allocate(cols, cols, nnz);
        SPAI_CUDA(cudaMemcpyAsync(out.ptr.get(), m_.ptr.data() + c0, sizeof(int64_t) * (cols + 1),
                                  cudaMemcpyDeviceToHost, ctx_.stream));
        DownloadWiden<T>(ctx_, m_.idx.data() + p0, m_.val.data() + p0, nnz, c0, out.idx.get(), out.val.get());
        ctx_.Sync();
        for (int64_t j = 0; j <= cols; ++j) out.ptr[j] -= p0;
        active[b] = 0;
        --live;
      }
      stopping.clear();
    };
    // AppendIteration (result_operations.cpp:53-67) for every live block
    auto append = [&](const std::vector<double>& residual) {
      fetch_counts();
      for (int64_t b = 0; b < blocks; ++b) {
        if (!active[b]) continue;
        SolveOutput& out = outputs[b];
        const double nb = static_cast<double>(offsets[b + 1] - offsets[b]);
        const double entries = nb * nb;
        SingleIterationData row;
        row.iteration = static_cast<int64_t>(out.history.size());
        out.iterations = row.iteration;
        row.residual_norm = residual[b];
        row.density_m = static_cast<double>(m_at[b + 1] - m_at[b]) / entries;
        row.density_direction = static_cast<double>(z_at[b + 1] - z_at[b]) / entries;
        out.history.push_back(row);
        if (row.residual_norm < opt_.tolerance) {
          out.converged = true;
          stopping.push_back(static_cast<int>(b));
        } else if (!opt_.dropping && opt_.max_density < 1.0 && row.density_m >= opt_.max_density) {
          stopping.push_back(static_cast<int>(b));
        }
      }
      snapshot();
    };
    // <Z, Pr A Z> and ||Pr A Z||^2 per block: the fused projection, reduced per block
    std::vector<double> num(static_cast<size_t>(blocks));
    std::vector<double> den(static_cast<size_t>(blocks));
    auto projection = [&]() {
      double* tt = ctx_.Partial(0, n_);
      double* bt = ctx_.Partial(1, n_);
      SpgemmExtras extras = AExtras();
      extras.row_scale = pr_vec_.data();
      extras.proj_tt = tt;
      extras.proj_bt = bt;
      DevCsc<T> unused;
      Spgemm(ctx_, A(), a_csr_, z_, unused, Epilogue::kProjection, extras);
      const double* parts[2] = {bt, tt};
      tree.Sums(ctx_, parts, 2, sums.data());
      for (int64_t b = 0; b < blocks; ++b) {
        num[b] = sums[b];
        den[b] = sums[blocks + b];
      }
    };

    // PrepareStateManager (methods_common.cpp:126-157) on every block
    Copy(ctx_, m0_, m_);
    for (DevCsc<T>* x : {&r_, &z_, &p_, &ap_, &az_, &tmp_, &q_}) Empty(*x);
    InvalidateResidualExtras();
    symmetric_ = true;
    if (opt_.dropping) {
      ApplyDroppingStrategy();
    } else {
      Residual();
    }
    std::vector<double> residual;
    residual_norms(residual);
    ComputeZ();
    append(residual);
    if (live > 0) projection();
    std::vector<double> alpha(static_cast<size_t>(blocks));
    DevCsc<T> scaled;
    for (int64_t i = 1; i <= opt_.max_iterations && live > 0; ++i) {
      for (int64_t b = 0; b < blocks; ++b) {
        alpha[b] = 0.0;
        if (!active[b]) continue;
        const double a = num[b] / den[b];
        if (!FiniteNonZeroHost(den[b]) || !std::isfinite(a)) {
          stopping.push_back(static_cast<int>(b));
        } else {
          alpha[b] = a;
        }
      }
      snapshot();
      if (live == 0) break;
      // M += alpha_b Z per block: Z scaled per column, then the union with
      // coefficient 1 (the same products and sums as the scalar union)
      SPAI_CUDA(cudaMemcpyAsync(alpha_dev.data(), alpha.data(), sizeof(double) * blocks, cudaMemcpyHostToDevice,
                                ctx_.stream));
      double* alpha_col = ColVec(0);
      BroadcastBlocksKernel<<<GridFor(n_, 256), 256, 0, ctx_.stream>>>(block_of_dev.data(), alpha_dev.data(), n_,
                                                                      alpha_col);
      SPAI_LAUNCH_CHECK();
      Copy(ctx_, z_, scaled);
      ScaleColumns(ctx_, scaled, alpha_col);
      Union(ctx_, m_, false, 1.0, scaled, 1.0, m_, UnionMode::kAxpby);
      UpdateResiduals([&] { Residual(); }, false);
      residual_norms(residual);
      append(residual);
      if (live == 0) break;
      ComputeZ();
      projection();
    }
    for (int64_t b = 0; b < blocks; ++b) {
      if (active[b]) stopping.push_back(static_cast<int>(b));
    }
    snapshot();
    ctx_.Sync();
  }

  int64_t iterations() const override { return iterations_; }
  int64_t m_nnz() const override { return m_.nnz; }
  int64_t n() const override { return n_; }
  const void* DeviceA() const override { return &A(); }
  const void* DeviceA64() const override { return &a64_; }

  void ExportMForPcg(void* csr_out, bool want_fp32) override {
    DevCsc<T> mt;
    Transpose(ctx_, m_, mt);
    if (want_fp32) {
      auto* out = static_cast<DevCsc<float>*>(csr_out);
      if constexpr (std::is_same<T, float>::value) {
        out->Swap(mt);
      } else {
        ConvertCsc(mt, *out);
      }
    } else {
      auto* out = static_cast<DevCsc<double>*>(csr_out);
      if constexpr (std::is_same<T, double>::value) {
        out->Swap(mt);
      } else {
        ConvertCsc(mt, *out);
      }
    }
  }

 private:
  template <class S, class D>
  void ConvertCsc(const DevCsc<S>& src, DevCsc<D>& dst) {
    dst.Shape(src.rows, src.cols, ctx_.stream);
    dst.ReserveNnz(src.nnz, ctx_.stream);
    SPAI_CUDA(cudaMemcpyAsync(dst.ptr.data(), src.ptr.data(), sizeof(int64_t) * (src.cols + 1),
                              cudaMemcpyDeviceToDevice, ctx_.stream));
    if (src.nnz > 0) {
      SPAI_CUDA(cudaMemcpyAsync(dst.idx.data(), src.idx.data(), sizeof(int32_t) * src.nnz, cudaMemcpyDeviceToDevice,
                                ctx_.stream));
      ConvertValues<S, D>(ctx_, src.val.data(), dst.val.data(), src.nnz);
    }
  }

  const DevCsc<T>& A() const {
    if constexpr (std::is_same<T, double>::value) {
      return a64_;
    } else {
      return a_;
    }
  }

  static bool IsFullDiagonal(const HostCsc& pr) {
    if (pr.nnz != pr.cols) return false;
    for (int64_t j = 0; j < pr.cols; ++j) {
      if (pr.ptr[j + 1] - pr.ptr[j] != 1 || pr.idx[pr.ptr[j]] != j) return false;
    }
    return true;
  }

  // Everything that follows from A in HBM (a64_ set): the FP32 copy, the
  // row-compressed copy, the ELL copies, the reference batches and ||A e_k||^2.
  void SetUpFromA() {
    if constexpr (!std::is_same<T, double>::value) {
      // the FP32 copy from the FP64 one already in HBM (same rounding as from the host values)
      ConvertCsc(a64_, a_);
    }
    Transpose(ctx_, A(), a_csr_);
    BuildAEll();
    if (ReferenceOrder()) InitReferenceBatches();
    // ||A e_k||^2 per column (methods_common.cpp:65-76)
    col_norm2_.Reserve(static_cast<size_t>(n_), ctx_.stream);
    if (opt_.dropping) {
      ColumnSquares(ctx_, View(a64_), col_norm2_.data());
    } else {
      SPAI_CUDA(cudaMemsetAsync(col_norm2_.data(), 0, sizeof(double) * n_, ctx_.stream));
    }
  }

  // Pr = diag(A)^-1 on the device, with the reference's messages for a bad diagonal.
  void DiagonalInversePreconditioner() {
    pr_vec_.Reserve(static_cast<size_t>(n_), ctx_.stream);
    int32_t* bad = ctx_.flags.data() + 4;
    SPAI_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), ctx_.stream));
    DiagonalInverseKernel<T><<<GridFor(n_, 256), 256, 0, ctx_.stream>>>(View(a64_), pr_vec_.data(), bad);
    SPAI_LAUNCH_CHECK();
    SPAI_CUDA(cudaMemcpyAsync(ctx_.host_flags + 4, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx_.stream));
    ctx_.Sync();
    if (ctx_.host_flags[4] & 1) throw std::invalid_argument("A has an invalid diagonal entry; provide Pr explicitly");
    if (ctx_.host_flags[4] & 2) {
      throw std::invalid_argument("A diagonal cannot be inverted safely; provide Pr explicitly");
    }
  }

  void IdentityM0() {
    m0_.Shape(n_, n_, ctx_.stream);
    m0_.ReserveNnz(n_, ctx_.stream);
    IdentityKernel<<<GridFor(n_ + 1, 256), 256, 0, ctx_.stream>>>(n_, m0_.ptr.data(), m0_.idx.data());
    SPAI_LAUNCH_CHECK();
    FillKernel<T><<<GridFor(n_, 256), 256, 0, ctx_.stream>>>(m0_.val.data(), n_, T(1));
    SPAI_LAUNCH_CHECK();
  }

  void CopyCheckedFromDevice(const DeviceCscInput& in, DevCsc<double>& out, const char* name) {
    UploadCheckedDeviceCsc(ctx_, in, out, name);
  }

  // ELL copies of A when no row or column of A holds more than kMaxEllWidth entries.
  void BuildAEll() {
    ell_width_ = 0;
    // the longest column of A and of its transpose (the longest row)
    unsigned long long* longest_dev = ctx_.select_state.data() + 3;
    SPAI_CUDA(cudaMemsetAsync(longest_dev, 0, sizeof(unsigned long long), ctx_.stream));
    LongestKernel<<<GridFor(n_, 256), 256, 0, ctx_.stream>>>(A().ptr.data(), a_csr_.ptr.data(), n_, longest_dev);
    SPAI_LAUNCH_CHECK();
    SPAI_CUDA(cudaMemcpyAsync(ctx_.host_counts + 2, longest_dev, sizeof(int64_t), cudaMemcpyDeviceToHost,
                              ctx_.stream));
    ctx_.Sync();
    const int64_t longest = ctx_.host_counts[2];
    a_longest_ = longest;
    if (longest > kMaxEllWidth) return;
    const int width = static_cast<int>(std::max<int64_t>(4, (longest + 3) / 4 * 4));
    const size_t slots = static_cast<size_t>(n_) * static_cast<size_t>(width);
    a_cols_ell_.Reserve(slots, ctx_.stream);
    a_rows_ell_.Reserve(slots, ctx_.stream);
    a_rows_ell_val_.Reserve(slots, ctx_.stream);
    BuildEll(ctx_, A(), width, a_cols_ell_.data(), static_cast<T*>(nullptr));
    BuildEll(ctx_, a_csr_, width, a_rows_ell_.data(), a_rows_ell_val_.data());
    ell_width_ = width;
  }

  SpgemmExtras AExtras() const {
    SpgemmExtras extras;
    if (ell_width_ > 0) {
      extras.x_cols_ell = a_cols_ell_.data();
      extras.x_rows_ell = a_rows_ell_.data();
      extras.x_rows_ell_val = a_rows_ell_val_.data();
      extras.ell_width = ell_width_;
    }
    return extras;
  }

  void Empty(DevCsc<T>& x) {
    x.Shape(n_, n_, ctx_.stream);
    x.ReserveNnz(0, ctx_.stream);
    FillZero(ctx_, x.ptr.data(), n_ + 1);
  }

  // ---- products (state_manager.cpp:47-66; dropping.cpp:97-104) ------------
  void MulA(const DevCsc<T>& in, DevCsc<T>& out) {
    Spgemm(ctx_, A(), a_csr_, in, out, opt_.dropping ? Epilogue::kPlain : Epilogue::kPruneZeros, AExtras());
  }

  void MulPr(const DevCsc<T>& in, DevCsc<T>& out) {
    if (pr_diagonal_) {
      DiagScale(ctx_, pr_vec_.data(), in, out, !opt_.dropping);
    } else {
      Spgemm(ctx_, pr_, pr_csr_, in, out, opt_.dropping ? Epilogue::kPlain : Epilogue::kPruneZeros);
    }
  }

  // R = I - A*M, with the per-column squares of R (for ||R||_F) and, when Pr
  // is diagonal and the dropping path keeps R's pattern, Z = Pr*R in the same pass.
  void Residual() {
    SpgemmExtras extras = AExtras();
    extras.col_squares = ctx_.Partial(kResidualPartial, n_);
    DevCsc<T>* z_out = nullptr;
    // the global methods (symmetric_) use Z = Pr*R right after every dropping-path residual
    if (pr_diagonal_ && opt_.dropping && symmetric_) {
      extras.row_scale = pr_vec_.data();
      z_out = &z_fused_;
    }
    const bool z_written = Spgemm(ctx_, A(), a_csr_, m_, r_, Epilogue::kResidual, extras, z_out);
    r_squares_ready_ = true;
    z_fused_ready_ = z_written;
  }

  void InvalidateResidualExtras() {
    r_squares_ready_ = false;
    z_fused_ready_ = false;
  }

  // Z = Pr*R: the copy fused into the last residual product when it is current.
  void ComputeZ() {
    if (z_fused_ready_) {
      z_.Swap(z_fused_);
      z_fused_ready_ = false;
      return;
    }
    MulPr(r_, z_);
  }

  // ---- reductions ----------------------------------------------------------
  double Dot(const DevCsc<T>& x, const DevCsc<T>& y) {
    if (ReferenceOrder()) return BatchTotal(BatchSums(&x, &y));
    double* part = ctx_.Partial(0, n_);
    ColumnDots(ctx_, View(x), View(y), part);
    const double* parts[1] = {part};
    TreeSums(ctx_, parts, 1, n_, 0);
    double out;
    FetchScalars(ctx_, 0, 1, &out);
    return out;
  }

  double SquaredNorm(const DevCsc<T>& x) {
    if (ReferenceOrder()) return BatchTotal(BatchSums(&x, nullptr));
    if (&x == &r_ && r_squares_ready_) {
      const double* ready[1] = {ctx_.Partial(kResidualPartial, n_)};
      TreeSums(ctx_, ready, 1, n_, 0);
      double out;
      FetchScalars(ctx_, 0, 1, &out);
      return out;
    }
    double* part = ctx_.Partial(0, n_);
    ColumnSquares(ctx_, View(x), part);
    const double* parts[1] = {part};
    TreeSums(ctx_, parts, 1, n_, 0);
    double out;
    FetchScalars(ctx_, 0, 1, &out);
    return out;
  }

  // ---- the reference's summation order (opt_.summation == 1) --------------
  bool ReferenceOrder() const { return opt_.summation == 1; }

  // InitializeBatches (methods_common.cpp:78-103): batch i holds columns
  // [n i / count, n (i + 1) / count) with count = min(n, num_threads).
  void InitReferenceBatches() {
    const int64_t count = std::min<int64_t>(n_, std::max<int64_t>(1, opt_.num_threads));
    batch_first_.assign(static_cast<size_t>(count + 1), 0);
    for (int64_t i = 0; i <= count; ++i) batch_first_[i] = n_ * i / count;
    std::vector<int32_t> batch_of(static_cast<size_t>(n_));
    for (int64_t b = 0; b < count; ++b) {
      for (int64_t j = batch_first_[b]; j < batch_first_[b + 1]; ++j) batch_of[j] = static_cast<int32_t>(b);
    }
    batch_first_dev_.Reserve(static_cast<size_t>(count + 1), ctx_.stream);
    batch_of_dev_.Reserve(static_cast<size_t>(n_), ctx_.stream);
    batch_sums_.Reserve(static_cast<size_t>(count), ctx_.stream);
    SPAI_CUDA(cudaMemcpyAsync(batch_first_dev_.data(), batch_first_.data(), sizeof(int64_t) * (count + 1),
                              cudaMemcpyHostToDevice, ctx_.stream));
    SPAI_CUDA(cudaMemcpyAsync(batch_of_dev_.data(), batch_of.data(), sizeof(int32_t) * n_, cudaMemcpyHostToDevice,
                              ctx_.stream));
    ctx_.Sync();
  }

  // Per-batch sums of squares of x (y null) or of the products x * y on the
  // common pattern, each sequential through its batch.
  std::vector<double> BatchSums(const DevCsc<T>* x, const DevCsc<T>* y) {
    const int64_t count = static_cast<int64_t>(batch_first_.size()) - 1;
    const int grid = GridFor(count, 64);
    if (y == nullptr) {
      BatchSquaresKernel<T><<<grid, 64, 0, ctx_.stream>>>(View(*x), batch_first_dev_.data(), count,
                                                          batch_sums_.data());
    } else {
      BatchDotsKernel<T><<<grid, 64, 0, ctx_.stream>>>(View(*x), View(*y), batch_first_dev_.data(), count,
                                                       batch_sums_.data());
    }
    SPAI_LAUNCH_CHECK();
    std::vector<double> out(static_cast<size_t>(count));
    SPAI_CUDA(cudaMemcpyAsync(out.data(), batch_sums_.data(), sizeof(double) * count, cudaMemcpyDeviceToHost,
                              ctx_.stream));
    ctx_.Sync();
    return out;
  }

  // the batches' partial sums added in batch order (the reference's reduction over batches)
  static double BatchTotal(const std::vector<double>& partial) {
    double total = 0.0;
    for (const double v : partial) total += v;
    return total;
  }

  // ---- sparse updates (sparse_operations.cpp:22-49) ------------------------
  void AddScaled(DevCsc<T>& t, const DevCsc<T>& d, double c) {
    if (&t == &r_) InvalidateResidualExtras();
    if (c != 0.0) {
      Union(ctx_, t, false, 1.0, d, c, t, UnionMode::kAxpby);
    } else {
      DropZeros(ctx_, t);
    }
  }

  void LinComb(const DevCsc<T>& x, double a, DevCsc<T>& y, double b) {
    Union(ctx_, y, true, b, x, a, y, UnionMode::kAxpby);
  }

  // state_manager.cpp:68-71
  int64_t MaxNonZeros() const {
    const double limit = opt_.max_density * static_cast<double>(n_) * static_cast<double>(n_);
    return std::max(n_, static_cast<int64_t>(std::floor(limit)));
  }

  // dropping.cpp:106-120
  void EnsureSymmetry() {
    if (!symmetric_) return;
    DevCsc<T> mt;
    Transpose(ctx_, m_, mt);
    Union(ctx_, m_, false, 1.0, mt, 1.0, m_, UnionMode::kHalfSum);
  }

  // dropping.cpp:122-175 (or the per-column top-k variant)
  void ApplyDroppingStrategy() {
    if (!SymmetrizeAndDrop(ctx_, m_, symmetric_, opt_.topk)) {
      // a column longer than the fused kernel takes: the same steps one pass each
      EnsureSymmetry();
      PruneColumnRelative(ctx_, m_);
      if (opt_.topk > 0) KeepTopKPerColumn(ctx_, m_, opt_.topk, true);
    }
    if (opt_.topk > 0) {
      Residual();
      return;
    }
    Residual();
    const int64_t budget = MaxNonZeros();
    const int64_t nonzeros = m_.nnz;
    if (nonzeros <= budget) return;
    DevBuf<double> tmp_values;
    DevBuf<double> scores;
    tmp_values.Reserve(static_cast<size_t>(nonzeros), ctx_.stream);
    scores.Reserve(static_cast<size_t>(nonzeros), ctx_.stream);
    // (A*R)(k, l) at every entry (k, l) of M: the masked product
    SpgemmMasked(ctx_, a_csr_, r_, m_, tmp_values.data());
    DropScores(ctx_, m_, col_norm2_.data(), tmp_values.data(), scores.data());
    GlobalDropByScore(ctx_, m_, scores.data(), true, nonzeros - budget);
    Residual();
  }

  // dropping.cpp:177-224 (or the per-column top-k variant)
  bool DropForMatrixType(DevCsc<T>& x) {
    if (!opt_.dropping) return false;
    const int64_t original = x.nnz;
    if (ReferenceOrder()) {
      // the reference prunes a direction per column batch, against that batch's norm (dropping.cpp:177-190)
      const std::vector<double> squares = BatchSums(&x, nullptr);
      std::vector<double> limit(squares.size());
      for (size_t b = 0; b < squares.size(); ++b) limit[b] = std::sqrt(squares[b]) * kEpsilon;
      batch_limit_.Reserve(limit.size(), ctx_.stream);
      SPAI_CUDA(cudaMemcpyAsync(batch_limit_.data(), limit.data(), sizeof(double) * limit.size(),
                                cudaMemcpyHostToDevice, ctx_.stream));
      double* column_limit = ColVec(1);
      BroadcastBlocksKernel<<<GridFor(n_, 256), 256, 0, ctx_.stream>>>(batch_of_dev_.data(), batch_limit_.data(),
                                                                      n_, column_limit);
      SPAI_LAUNCH_CHECK();
      PruneAbsAtMostPerColumn(ctx_, x, column_limit);
    } else {
      const double limit = std::sqrt(SquaredNorm(x)) * kEpsilon;
      PruneAbsAtMost(ctx_, x, limit);
    }
    if (opt_.topk > 0) {
      KeepTopKPerColumn(ctx_, x, opt_.topk, false);
      return x.nnz != original;
    }
    const int64_t budget = MaxNonZeros();
    if (x.nnz <= budget) return x.nnz != original;
    DevBuf<double> scores;
    scores.Reserve(static_cast<size_t>(x.nnz), ctx_.stream);
    AbsScores(ctx_, x, scores.data());
    GlobalDropByScore(ctx_, x, scores.data(), false, x.nnz - budget);
    return true;
  }

  // state_manager.cpp:81-95
  void StabilizeResiduals() {
    const double norm = std::sqrt(SquaredNorm(r_));
    const double floor = 64.0 * kEpsilon * std::sqrt(static_cast<double>(n_));
    const double limit = std::max(10.0 * opt_.tolerance, floor);
    if (std::isfinite(norm) && norm > limit) return;
    Residual();
  }

  // methods_common.hpp:83-93
  template <class F>
  void UpdateResiduals(F recursive_update, bool stabilize) {
    if (opt_.dropping) {
      ApplyDroppingStrategy();
      return;
    }
    recursive_update();
    if (stabilize) StabilizeResiduals();
  }

  // result_operations.cpp:53-67
  bool AppendIteration(const DevCsc<T>& direction) {
    const int64_t iter = static_cast<int64_t>(history_.size());
    iterations_ = iter;
    const double residual = history_.empty() ? initial_residual_ : std::sqrt(SquaredNorm(r_));
    const double entries = static_cast<double>(n_) * static_cast<double>(n_);
    SingleIterationData row;
    row.iteration = iter;
    row.residual_norm = residual;
    row.density_m = static_cast<double>(m_.nnz) / entries;
    row.density_direction = static_cast<double>(direction.nnz) / entries;
    history_.push_back(row);
    if (row.residual_norm < opt_.tolerance) {
      converged_ = true;
      return true;
    }
    return !opt_.dropping && opt_.max_density < 1.0 && row.density_m >= opt_.max_density;
  }

  static bool FiniteNonZeroHost(double v) { return std::isfinite(v) && std::fabs(v) > 0.0; }

  // ---- Global CG (conjugate_gradient.cpp:15-83) ----------------------------
  void RunCg() {
    ComputeZ();
    Copy(ctx_, z_, p_);
    double r_z = Dot(r_, z_);
    DropForMatrixType(p_);
    if (AppendIteration(p_)) return;
    MulA(p_, ap_);
    for (int64_t i = 1; i <= opt_.max_iterations; ++i) {
      const double den = Dot(p_, ap_);
      if (!FiniteNonZeroHost(r_z) || !FiniteNonZeroHost(den)) break;
      const double alpha = r_z / den;
      if (!std::isfinite(alpha)) break;
      const double previous = r_z;
      AddScaled(m_, p_, alpha);
      UpdateResiduals([&] { AddScaled(r_, ap_, -alpha); }, false);
      if (AppendIteration(p_)) break;
      ComputeZ();
      r_z = Dot(r_, z_);
      const double beta = r_z / previous;
      if (!std::isfinite(beta)) break;
      LinComb(z_, 1.0, p_, beta);
      DropForMatrixType(p_);
      MulA(p_, ap_);
    }
  }

  // num = <Z, Pr A Z>, den = ||Pr A Z||^2 (minimal_residual.cpp:44-52,78-88)
  void MrProjection(double& num, double& den) {
    if (pr_diagonal_ && !ReferenceOrder()) {
      double* tt = ctx_.Partial(0, n_);
      double* bt = ctx_.Partial(1, n_);
      SpgemmExtras extras = AExtras();
      extras.row_scale = pr_vec_.data();
      extras.proj_tt = tt;
      extras.proj_bt = bt;
      DevCsc<T> unused;
      Spgemm(ctx_, A(), a_csr_, z_, unused, Epilogue::kProjection, extras);
      const double* parts[2] = {bt, tt};
      TreeSums(ctx_, parts, 2, n_, 0);
      double out[2];
      FetchScalars(ctx_, 0, 2, out);
      num = out[0];
      den = out[1];
      return;
    }
    MulA(z_, az_);
    MulPr(az_, tmp_);
    num = Dot(z_, tmp_);
    den = SquaredNorm(tmp_);
  }

  // ---- Global MR (minimal_residual.cpp:31-93) ------------------------------
  void RunMr() {
    ComputeZ();
    if (AppendIteration(z_)) return;
    double num = 0.0;
    double den = 0.0;
    MrProjection(num, den);
    if (FusedEligible()) {
      // iterations 1.. as one CUDA graph of fused kernels (mr_fused.cu): same arithmetic, same bits
      if (opt_.max_iterations < 1 || !FiniteNonZeroHost(den)) return;
      const double alpha = num / den;
      if (!std::isfinite(alpha)) return;
      FusedMrProblem problem;
      problem.n = n_;
      problem.topk = static_cast<int>(opt_.topk);
      problem.a_nnz = a64_.nnz;
      problem.a_longest = a_longest_;
      problem.ell_width = ell_width_;
      problem.a_cols_ell = a_cols_ell_.data();
      problem.a_rows_ell = a_rows_ell_.data();
      problem.a_rows_ell_val = a_rows_ell_val_.data();
      problem.pr = pr_vec_.data();
      problem.max_iterations = opt_.max_iterations;
      problem.tolerance = opt_.tolerance;
      if (FusedMrApplicable(problem)) {
        if (!fused_) fused_ = MakeFusedMr<T>();
        const FusedMrOutcome outcome = fused_->Run(ctx_, problem, &m_, &z_, alpha, history_);
        if (outcome.ran) {
          if (outcome.overflow) {
            fused_overflowed_ = true;
            return;
          }
          iterations_ = outcome.iterations;
          converged_ = outcome.converged;
          return;
        }
      }
    }
    for (int64_t i = 1; i <= opt_.max_iterations; ++i) {
      if (!FiniteNonZeroHost(den)) break;
      const double alpha = num / den;
      if (!std::isfinite(alpha)) break;
      AddScaled(m_, z_, alpha);
      UpdateResiduals([&] { Residual(); }, false);
      if (AppendIteration(z_)) break;
      ComputeZ();
      MrProjection(num, den);
    }
  }

  // ---- Global LOMR (locally_minimal_residual.cpp:54-118) -------------------
  void RunLomr() {
    ComputeZ();
    if (AppendIteration(z_)) return;
    for (int64_t i = 1; i <= opt_.max_iterations; ++i) {
      MulA(p_, ap_);
      MulA(z_, az_);
      MulPr(az_, tmp_);
      double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      if (ReferenceOrder()) {
        s[0] = Dot(az_, tmp_);
        s[1] = Dot(z_, az_);
        if (i > 1) {
          MulPr(ap_, tmp_);
          s[2] = Dot(ap_, tmp_);
          s[3] = Dot(az_, tmp_);
          s[4] = Dot(z_, ap_);
        }
      } else {
        double* parts_buf[5];
        for (int k = 0; k < 5; ++k) parts_buf[k] = ctx_.Partial(k, n_);
        ColumnDots(ctx_, View(az_), View(tmp_), parts_buf[0]);
        ColumnDots(ctx_, View(z_), View(az_), parts_buf[1]);
        int arrays = 2;
        if (i > 1) {
          MulPr(ap_, tmp_);
          ColumnDots(ctx_, View(ap_), View(tmp_), parts_buf[2]);
          ColumnDots(ctx_, View(az_), View(tmp_), parts_buf[3]);
          ColumnDots(ctx_, View(z_), View(ap_), parts_buf[4]);
          arrays = 5;
        }
        const double* parts[5] = {parts_buf[0], parts_buf[1], parts_buf[2], parts_buf[3], parts_buf[4]};
        TreeSums(ctx_, parts, arrays, n_, 0);
        FetchScalars(ctx_, 0, arrays, s);
      }
      const double az_praz = s[0];
      const double z_az = s[1];
      const double ap_prap = s[2];
      const double az_prap = s[3];
      const double z_ap = s[4];
      double delta;
      double gamma;
      if (i == 1) {
        if (!FiniteNonZeroHost(az_praz)) break;
        delta = z_az / az_praz;
        gamma = 1.0;
      } else {
        const double gram[4] = {az_praz, az_prap, az_prap, ap_prap};
        const double rhs[2] = {z_az, z_ap};
        double coef[2];
        SolveLeastSquares2x2(gram, rhs, coef);
        delta = coef[0];
        gamma = coef[1];
      }
      if (!std::isfinite(delta) || !std::isfinite(gamma)) break;
      AddScaled(m_, z_, delta);
      AddScaled(m_, p_, gamma);
      UpdateResiduals(
          [&] {
            AddScaled(r_, az_, -delta);
            AddScaled(r_, ap_, -gamma);
          },
          false);
      const double ratio = delta != 0.0 ? gamma / delta : 0.0;
      LinComb(z_, 1.0, p_, std::isfinite(ratio) ? ratio : 0.0);
      DropForMatrixType(p_);
      if (AppendIteration(p_)) break;
      ComputeZ();
    }
  }

  // ---- Inner-Outer (inner_outer_common.hpp:14-107) -------------------------
  void RunInnerOuter(bool locally_optimal) {
    if (AppendIteration(p_)) return;
    double* normalization = ColVec(5);
    const int grid = GridFor(n_, 128);
    FillKernel<double><<<GridFor(n_, 256), 256, 0, ctx_.stream>>>(normalization, n_, 1.0);
    SPAI_LAUNCH_CHECK();
    DevCsc<T> outer;
    DevCsc<T> outer_csr;
    for (int64_t iteration = 0; iteration < opt_.max_iterations;) {
      Copy(ctx_, m_, outer);
      Transpose(ctx_, outer, outer_csr);
      Residual();
      Empty(q_);
      const int64_t inner_count = std::min(opt_.inner_iterations, opt_.max_iterations - iteration);
      for (int64_t inner = 0; inner < inner_count; ++inner, ++iteration) {
        Spgemm(ctx_, outer, outer_csr, r_, z_, opt_.dropping ? Epilogue::kPlain : Epilogue::kPruneZeros);
        MulA(z_, az_);
        if (locally_optimal) {
          Spgemm(ctx_, A(), a_csr_, q_, ap_, Epilogue::kPlain, AExtras());
        }
        double* r_az = ctx_.Partial(0, n_);
        double* az_az = ctx_.Partial(1, n_);
        double* az_aq = ctx_.Partial(2, n_);
        double* aq_aq = ctx_.Partial(3, n_);
        double* r_aq = ctx_.Partial(4, n_);
        ColumnDots(ctx_, View(r_), View(az_), r_az);
        ColumnSquares(ctx_, View(az_), az_az);
        const bool first = !locally_optimal || inner == 0;
        if (!first) {
          ColumnDots(ctx_, View(az_), View(ap_), az_aq);
          ColumnSquares(ctx_, View(ap_), aq_aq);
          ColumnDots(ctx_, View(r_), View(ap_), r_aq);
        }
        double* delta = ColVec(0);
        double* gamma = ColVec(1);
        InnerOuterStepKernel<<<grid, 128, 0, ctx_.stream>>>(n_, r_az, az_az, az_aq, aq_aq, r_aq, locally_optimal,
                                                            first, delta, gamma, normalization);
        SPAI_LAUNCH_CHECK();
        Copy(ctx_, z_, p_);
        ScaleColumns(ctx_, p_, delta);
        if (locally_optimal) {
          ScaleColumns(ctx_, q_, gamma);
          AddScaled(p_, q_, 1.0);
        }
        const bool dropped = DropForMatrixType(p_);
        MulA(p_, ap_);
        if (dropped) {
          double* num = ctx_.Partial(0, n_);
          double* den = ctx_.Partial(1, n_);
          double* correction = ColVec(2);
          ColumnDots(ctx_, View(r_), View(ap_), num);
          ColumnSquares(ctx_, View(ap_), den);
          SafeQuotientKernel<<<grid, 128, 0, ctx_.stream>>>(n_, num, den, correction);
          SPAI_LAUNCH_CHECK();
          ScaleColumns(ctx_, p_, correction);
          ScaleColumns(ctx_, ap_, correction);
        }
        AddScaled(m_, p_, 1.0);
        if (locally_optimal) {
          Copy(ctx_, p_, q_);
          ScaleColumns(ctx_, q_, normalization);
        }
        UpdateResiduals([&] { AddScaled(r_, ap_, -1.0); }, true);
        if (AppendIteration(p_)) return;
      }
    }
  }

  // Global MR with per-column top-k, a diagonal Pr and ELL copies of A, in the device order.
  bool FusedEligible() const {
    return FusedMrEnabled() && fused_allowed_ && opt_.method == Method::kGlobalMr && opt_.dropping &&
           opt_.topk > 0 && pr_diagonal_ && !ReferenceOrder() && ell_width_ > 0 && symmetric_;
  }

  double* ColVec(int i) {
    ctx_.colvec[i].Reserve(static_cast<size_t>(n_), ctx_.stream);
    return ctx_.colvec[i].data();
  }

  Ctx& ctx_;
  SolveOptions opt_;
  int64_t n_ = 0;
  bool symmetric_ = true;
  DevCsc<double> a64_;
  DevCsc<T> a_;  // FP32 copy of A in mixed precision (unused in FP64)
  DevCsc<T> a_csr_;
  DevBuf<double> col_norm2_;
  bool pr_diagonal_ = true;
  DevBuf<T> pr_vec_;
  DevCsc<T> pr_;
  DevCsc<T> pr_csr_;
  DevCsc<T> m0_;
  DevCsc<T> m_, r_, z_, p_, ap_, az_, tmp_, q_;
  // fixed-width copies of A for the SpGEMM column kernel (stencil-like A only)
  DevBuf<int32_t> a_cols_ell_;
  DevBuf<int32_t> a_rows_ell_;
  DevBuf<T> a_rows_ell_val_;
  int ell_width_ = 0;
  int64_t a_longest_ = 0;  // longest column or row of A
  static constexpr int kMaxEllWidth = 16;
  std::unique_ptr<FusedMrBase> fused_;
  bool fused_allowed_ = true;
  bool fused_overflowed_ = false;
  DevCsc<T> z_fused_;             // Pr*R written by the last residual product
  bool r_squares_ready_ = false;  // Partial(kResidualPartial) holds R's column squares
  bool z_fused_ready_ = false;
  static constexpr int kResidualPartial = 7;
  std::vector<int64_t> batch_first_;  // reference order: first column of every batch, then n
  DevBuf<int64_t> batch_first_dev_;
  DevBuf<int32_t> batch_of_dev_;      // batch of every column
  DevBuf<double> batch_sums_;
  DevBuf<double> batch_limit_;
  std::vector<SingleIterationData> history_;
  double initial_residual_ = 0.0;
  int64_t iterations_ = 0;
  bool converged_ = false;
};

}  // namespace

std::unique_ptr<SolverBase> MakeSolver(Ctx& ctx, const SolveOptions& options) {
  if (options.precision == 0) return std::unique_ptr<SolverBase>(new Solver<double>(ctx, options));
  return std::unique_ptr<SolverBase>(new Solver<float>(ctx, options));
}

namespace {
// True when pred(i) holds for every i in [0, n); large ranges are split over host threads.
template <class Pred>
bool AllOf(int64_t n, Pred pred) {
  const int64_t parts = n < (int64_t{1} << 20) ? 1 : std::min<int64_t>(8, std::max(1u, std::thread::hardware_concurrency()));
  if (parts <= 1) {
    for (int64_t i = 0; i < n; ++i) {
      if (!pred(i)) return false;
    }
    return true;
  }
  std::atomic<bool> ok{true};
  std::vector<std::thread> pool;
  for (int64_t k = 0; k < parts; ++k) {
    pool.emplace_back([&, k]() {
      const int64_t last = n * (k + 1) / parts;
      for (int64_t i = n * k / parts; i < last && ok.load(std::memory_order_relaxed); ++i) {
        if (!pred(i)) ok.store(false, std::memory_order_relaxed);
      }
    });
  }
  for (auto& t : pool) t.join();
  return ok.load();
}
}  // namespace

HostCsc CheckedMatrix(const MatrixData& data) {
  // GetCompressedSparseMatrix (methods_c_api.cpp:16-40)
  if (data.rows <= 0 || data.cols <= 0 || data.nnz <= 0) {
    throw std::invalid_argument("Sparse matrix dimensions and nnz must be positive");
  }
  if (!AllOf(data.cols, [&](int64_t i) { return data.col_offsets[i] <= data.col_offsets[i + 1]; })) {
    throw std::invalid_argument("Sparse matrix column offsets must be non-decreasing");
  }
  if (!AllOf(data.nnz, [&](int64_t i) { return data.row_indices[i] >= 0 && data.row_indices[i] < data.rows; })) {
    throw std::invalid_argument("Sparse matrix row idx is out of range");
  }
  if (data.rows > static_cast<int64_t>(std::numeric_limits<int32_t>::max()) ||
      data.cols > static_cast<int64_t>(std::numeric_limits<int32_t>::max())) {
    throw std::invalid_argument("Sparse matrix dimensions exceed the 32-bit row index range of the device layout");
  }
  HostCsc h;
  h.rows = data.rows;
  h.cols = data.cols;
  h.nnz = data.nnz;
  h.ptr = data.col_offsets;
  h.idx = data.row_indices;
  h.val = data.values;
  return h;
}

void ValidateProblem(const HostCsc& a, const HostCsc* m0, const HostCsc* pr, const MethodParams& p) {
  // methods_common.cpp:12-36
  if (a.rows != a.cols || a.rows == 0) throw std::invalid_argument("A must be a non-empty square matrix");
  if (m0 != nullptr && (m0->rows != a.rows || m0->cols != a.cols)) {
    throw std::invalid_argument("Initial preconditioner M0 must have the same shape as A");
  }
  if (pr != nullptr && (pr->rows != a.rows || pr->cols != a.cols)) {
    throw std::invalid_argument("Pr must have the same shape as A");
  }
  if (p.max_iterations <= 0) throw std::invalid_argument("max_iterations must be positive");
  if (!std::isfinite(p.tolerance) || p.tolerance < 0.0) {
    throw std::invalid_argument("tolerance must be finite and non-negative");
  }
  if (!std::isfinite(p.max_density) || p.max_density <= kMinDensity || p.max_density > 1.0) {
    throw std::invalid_argument("max_density must be finite and in the interval (0, 1]");
  }
  const double entries = p.max_density * static_cast<double>(a.rows) * static_cast<double>(a.rows);
  if (p.enable_dropping != 0 && entries < static_cast<double>(a.rows)) {
    throw std::invalid_argument("max_density is too small to preserve the diagonal of M");
  }
  // methods_common.cpp:38-48
  if (p.num_threads <= 0) throw std::invalid_argument("Invalid threads count value");
}

}  // namespace spai
