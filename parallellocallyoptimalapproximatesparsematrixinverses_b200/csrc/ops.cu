// Sparse-matrix building blocks on sm_100a: scans, the canonical reduction
// tree, unions, filters (pruning, top-k, global cutoff), transposition and
// radix selection.  All are HBM-bound integer/byte work plus light FP64
// arithmetic; none is a contraction, so none uses tensor cores.

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <limits>

#include "device.cuh"
#include "ops.cuh"
#include "profile.cuh"
#include "tree.cuh"

namespace spai {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int64_t kScanTile = kScanThreads * kScanItems;

constexpr double kDblEps = 2.220446049250313080847e-16;

__device__ __forceinline__ unsigned LaneMaskLt() {
  unsigned mask;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(mask));
  return mask;
}

// ---------------------------------------------------------------------------
// Scan
__global__ void ScanTileKernel(const int64_t* __restrict__ in, int64_t n, int64_t* __restrict__ out,
                               int64_t* __restrict__ tile_sums) {
  __shared__ int64_t warp_sums[kScanThreads / kWarp];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + static_cast<int64_t>(threadIdx.x) * kScanItems;
  int64_t v[kScanItems];
  int64_t local = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t at = base + i;
    v[i] = at < n ? in[at] : 0;
    local += v[i];
  }
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int64_t inclusive = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, inclusive, o);
    if (lane >= o) inclusive += y;
  }
  if (lane == 31) warp_sums[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    int64_t w = lane < kScanThreads / kWarp ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / kWarp) warp_sums[lane] = w;
  }
  __syncthreads();
  int64_t running = inclusive - local + (warp > 0 ? warp_sums[warp - 1] : 0);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    running += v[i];
    if (base + i < n) out[base + i + 1] = running;
  }
  if (threadIdx.x == kScanThreads - 1) tile_sums[blockIdx.x] = running;
}

__global__ void ScanAddKernel(int64_t n, int64_t* __restrict__ out, const int64_t* __restrict__ tile_prefix) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i == 0) out[0] = 0;
  if (i < n) out[i + 1] += tile_prefix[i / kScanTile];
}

void ScanRecursive(Ctx& ctx, const int64_t* in, int64_t n, int64_t* out, DevBuf<int64_t>& scratch, size_t offset) {
  const int64_t tiles = CeilDiv(n, kScanTile);
  int64_t* tile_sums = scratch.data() + offset;
  ScanTileKernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, ctx.stream>>>(in, n, out, tile_sums);
  SPAI_LAUNCH_CHECK();
  if (tiles > 1) {
    int64_t* tile_prefix = tile_sums + tiles;
    ScanRecursive(ctx, tile_sums, tiles, tile_prefix, scratch, offset + 2 * tiles + 1);
    ScanAddKernel<<<static_cast<unsigned>(CeilDiv(n, 256)), 256, 0, ctx.stream>>>(n, out, tile_prefix);
    SPAI_LAUNCH_CHECK();
  } else {
    SPAI_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), ctx.stream));
  }
}

// ---------------------------------------------------------------------------
// Canonical tree: 256 lanes per 4096-value chunk, then a butterfly.
struct TreeArgs {
  const double* src[8];
  const double* src2[8];  // when set, level-one terms are src[i] * src2[i]
};

// The lanes' partial sums of one chunk -> the chunk's sum (tree.cuh).
__device__ __forceinline__ double ChunkButterfly(double s, double* shared) { return TreeButterfly(s, shared); }

__global__ void TreeChunkKernel(TreeArgs args, int64_t n, double* __restrict__ out, int64_t out_stride) {
  __shared__ double shared[kTreeLanes];
  const double* __restrict__ src = args.src[blockIdx.y];
  const double* __restrict__ src2 = args.src2[blockIdx.y];
  const int t = threadIdx.x;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTreeChunk + t;
  double s = 0.0;
  if (src2 != nullptr) {
#pragma unroll
    for (int m = 0; m < static_cast<int>(kTreeChunk / kTreeLanes); ++m) {
      const int64_t i = base + static_cast<int64_t>(kTreeLanes) * m;
      if (i < n) s = Add(s, Mul(src[i], src2[i]));
    }
  } else {
#pragma unroll
    for (int m = 0; m < static_cast<int>(kTreeChunk / kTreeLanes); ++m) {
      const int64_t i = base + static_cast<int64_t>(kTreeLanes) * m;
      if (i < n) s = Add(s, src[i]);
    }
  }
  s = ChunkButterfly(s, shared);
  if (t == 0) out[blockIdx.y * out_stride + blockIdx.x] = s;
}

// One level of the tree over many segments at once.  Block b sums
// src[start[b], end[b]) (at most one chunk, lanes as TreeChunkKernel) into
// out[dst[b]]; table = start[blocks] | end[blocks] | dst[blocks].
__global__ void SegmentChunkKernel(TreeArgs args, const int64_t* __restrict__ table, int64_t blocks,
                                   double* __restrict__ out, int64_t out_stride) {
  __shared__ double shared[kTreeLanes];
  const double* __restrict__ src = args.src[blockIdx.y];
  const int t = threadIdx.x;
  const int64_t start = table[blockIdx.x];
  const int64_t end = table[blocks + blockIdx.x];
  double s = 0.0;
#pragma unroll
  for (int m = 0; m < static_cast<int>(kTreeChunk / kTreeLanes); ++m) {
    const int64_t i = start + t + static_cast<int64_t>(kTreeLanes) * m;
    if (i < end) s = Add(s, src[i]);
  }
  s = ChunkButterfly(s, shared);
  if (t == 0) out[blockIdx.y * out_stride + table[2 * blocks + blockIdx.x]] = s;
}

// ---------------------------------------------------------------------------
// Per-column partial sums
template <class T>
__global__ void ColumnSquaresKernel(CscView<T> x, double* __restrict__ partial) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < x.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int64_t p = x.ptr[j]; p < x.ptr[j + 1]; ++p) {
      const double v = static_cast<double>(x.val[p]);
      s = Add(s, Mul(v, v));
    }
    partial[j] = s;
  }
}

template <class T>
__global__ void ColumnDotsKernel(CscView<T> x, CscView<T> y, double* __restrict__ partial) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < x.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    int64_t p = x.ptr[j];
    int64_t q = y.ptr[j];
    const int64_t pe = x.ptr[j + 1];
    const int64_t qe = y.ptr[j + 1];
    while (p < pe && q < qe) {
      const int32_t a = x.idx[p];
      const int32_t b = y.idx[q];
      if (a == b) {
        s = Add(s, Mul(static_cast<double>(x.val[p]), static_cast<double>(y.val[q])));
        ++p;
        ++q;
      } else if (a < b) {
        ++p;
      } else {
        ++q;
      }
    }
    partial[j] = s;
  }
}

// ---------------------------------------------------------------------------
// Union (thread per column, two phases)
// Values in the storage type's arithmetic (FP64 for double, FP32 for float storage).
template <class T>
__device__ __forceinline__ T UnionBoth(T y, T x, bool scale_y, T ys, T xs, int mode) {
  if (mode == static_cast<int>(UnionMode::kHalfSum)) return Mul(T(0.5), Add(y, x));
  const T yv = scale_y ? Mul(ys, y) : y;
  return Add(yv, Mul(xs, x));
}

template <class T>
__device__ __forceinline__ T UnionLeft(T y, bool scale_y, T ys, int mode) {
  if (mode == static_cast<int>(UnionMode::kHalfSum)) return Mul(T(0.5), Add(y, T(0)));
  const T yv = scale_y ? Mul(ys, y) : y;
  return Add(yv, T(0));
}

template <class T>
__device__ __forceinline__ T UnionRight(T x, T xs, int mode) {
  if (mode == static_cast<int>(UnionMode::kHalfSum)) return Mul(T(0.5), Add(T(0), x));
  return Add(T(0), Mul(xs, x));
}

// One thread per column: used for columns whose X part is longer than the
// warp kernels' cap (min_nx); prunes exact zeros inline.
template <class T, bool kWrite>
__global__ void UnionKernel(CscView<T> y, CscView<T> x, bool scale_y, double ys, double xs, int mode, int64_t min_nx,
                            int64_t* __restrict__ counts, const int64_t* __restrict__ out_ptr,
                            int32_t* __restrict__ out_idx, T* __restrict__ out_val) {
  const bool prune = mode == static_cast<int>(UnionMode::kAxpby);
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < y.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (x.ptr[j + 1] - x.ptr[j] <= min_nx) continue;
    int64_t p = y.ptr[j];
    int64_t q = x.ptr[j];
    const int64_t pe = y.ptr[j + 1];
    const int64_t qe = x.ptr[j + 1];
    int64_t o = kWrite ? out_ptr[j] : 0;
    int64_t count = 0;
    const T yst = static_cast<T>(ys);
    const T xst = static_cast<T>(xs);
    while (p < pe || q < qe) {
      int32_t row;
      T stored;
      if (p < pe && q < qe && y.idx[p] == x.idx[q]) {
        row = y.idx[p];
        stored = UnionBoth<T>(y.val[p], x.val[q], scale_y, yst, xst, mode);
        ++p;
        ++q;
      } else if (p < pe && (q >= qe || y.idx[p] < x.idx[q])) {
        row = y.idx[p];
        stored = UnionLeft<T>(y.val[p], scale_y, yst, mode);
        ++p;
      } else {
        row = x.idx[q];
        stored = UnionRight<T>(x.val[q], xst, mode);
        ++q;
      }
      if (prune && stored == T(0)) continue;
      if (kWrite) {
        out_idx[o] = row;
        out_val[o] = stored;
        ++o;
      } else {
        ++count;
      }
    }
    if (!kWrite) counts[j] = count;
  }
}

// ---------------------------------------------------------------------------
// Warp-per-column filters
template <class T>
struct KeepNonZero {
  __device__ void Begin(const CscView<T>&, int64_t, int) {}
  __device__ bool Keep(int64_t, int64_t, int32_t, T v) const {
    const double d = static_cast<double>(v);
    return !(fabs(d) <= 0.0);
  }
};

template <class T>
struct KeepAboveLimit {
  double limit;
  const double* column_limit = nullptr;  // when set: the limit of each column
  __device__ void Begin(const CscView<T>&, int64_t col, int) {
    if (column_limit != nullptr) limit = column_limit[col];
  }
  __device__ bool Keep(int64_t, int64_t, int32_t, T v) const {
    return !(fabs(static_cast<double>(v)) <= limit);
  }
};

template <class T>
struct KeepColumnRelative {
  double threshold = 0.0;
  __device__ void Begin(const CscView<T>& x, int64_t col, int lane) {
    double s = 0.0;
    if (lane == 0) {
      for (int64_t p = x.ptr[col]; p < x.ptr[col + 1]; ++p) {
        const double v = static_cast<double>(x.val[p]);
        s = Add(s, Mul(v, v));
      }
      s = Mul(kDblEps, sqrt(s));
    }
    threshold = __shfl_sync(0xffffffffu, s, 0);
  }
  __device__ bool Keep(int64_t col, int64_t, int32_t row, T v) const {
    const double d = static_cast<double>(v);
    return d != 0.0 && (static_cast<int64_t>(row) == col || fabs(d) >= threshold);
  }
};

// (|v|, row) keys; keeps the largest `k` (diagonal protected if asked).
template <class T>
struct KeepTopK {
  int64_t k;
  bool protect;
  bool keep_all = true;
  double cut_abs = 0.0;
  int32_t cut_row = 0;
  __device__ void Begin(const CscView<T>& x, int64_t col, int lane) {
    const int64_t start = x.ptr[col];
    const int64_t end = x.ptr[col + 1];
    const int64_t count = end - start;
    keep_all = count <= k;
    if (keep_all) return;
    // candidates: all entries except a protected diagonal
    bool has_diag = false;
    if (protect) {
      for (int64_t base = start; base < end; base += kWarp) {
        const int64_t p = base + lane;
        const bool d = p < end && static_cast<int64_t>(x.idx[p]) == col;
        if (__any_sync(0xffffffffu, d)) has_diag = true;
      }
    }
    const int64_t candidates = count - (has_diag ? 1 : 0);
    const int64_t keep_off = k - (has_diag ? 1 : 0) > 0 ? k - (has_diag ? 1 : 0) : 0;
    const int64_t drop = candidates - keep_off;
    if (drop <= 0) {
      keep_all = true;
      return;
    }
    // the drop-th smallest candidate key is the cutoff
    double found_abs = 0.0;
    int32_t found_row = 0;
    bool found = false;
    for (int64_t base = start; base < end; base += kWarp) {
      const int64_t p = base + lane;
      bool mine = false;
      double a = 0.0;
      int32_t r = 0;
      if (p < end) {
        r = x.idx[p];
        a = fabs(static_cast<double>(x.val[p]));
        const bool is_cand = !(protect && static_cast<int64_t>(r) == col);
        if (is_cand) {
          int64_t rank = 0;
          for (int64_t q = start; q < end; ++q) {
            const int32_t rq = x.idx[q];
            if (protect && static_cast<int64_t>(rq) == col) continue;
            const double aq = fabs(static_cast<double>(x.val[q]));
            rank += (aq < a || (aq == a && rq < r)) ? 1 : 0;
          }
          mine = rank == drop - 1;
        }
      }
      const unsigned ballot = __ballot_sync(0xffffffffu, mine);
      if (ballot != 0u) {
        const int src = __ffs(ballot) - 1;
        found_abs = __shfl_sync(0xffffffffu, a, src);
        found_row = __shfl_sync(0xffffffffu, r, src);
        found = true;
      }
    }
    cut_abs = found_abs;
    cut_row = found_row;
    if (!found) keep_all = true;
  }
  __device__ bool Keep(int64_t col, int64_t, int32_t row, T v) const {
    if (keep_all) return true;
    if (protect && static_cast<int64_t>(row) == col) return true;
    const double a = fabs(static_cast<double>(v));
    return a > cut_abs || (a == cut_abs && row > cut_row);
  }
};

__device__ __forceinline__ unsigned long long OrderedBits(double s) {
  if (s == 0.0) s = 0.0;  // -0.0 and +0.0 compare equal in the reference ordering
  unsigned long long u = static_cast<unsigned long long>(__double_as_longlong(s));
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

// keep iff diagonal (when skipped) or (ordered score, offset) > cutoff.
template <class T>
struct KeepAboveCutoff {
  const double* scores;
  const int64_t* column_base;  // first candidate offset of each column
  const unsigned long long* cutoff;  // [score bits, offset]
  bool skip_diag;
  int64_t diag_pos = -1;
  int64_t start = 0;
  unsigned long long cut_score = 0;
  unsigned long long cut_offset = 0;
  __device__ void Begin(const CscView<T>& x, int64_t col, int lane) {
    start = x.ptr[col];
    const int64_t end = x.ptr[col + 1];
    cut_score = cutoff[0];
    cut_offset = cutoff[1];
    diag_pos = -1;
    if (skip_diag) {
      for (int64_t base = start; base < end; base += kWarp) {
        const int64_t p = base + lane;
        const bool d = p < end && static_cast<int64_t>(x.idx[p]) == col;
        const unsigned b = __ballot_sync(0xffffffffu, d);
        if (b != 0u) diag_pos = base + __ffs(b) - 1;
      }
    }
  }
  __device__ bool Keep(int64_t col, int64_t pos, int32_t row, T) const {
    if (skip_diag && static_cast<int64_t>(row) == col) return true;
    const int64_t offset = skip_diag ? column_base[col] + (pos - start) - ((diag_pos >= 0 && diag_pos < pos) ? 1 : 0)
                                     : pos;
    const unsigned long long s = OrderedBits(scores[pos]);
    const unsigned long long o = static_cast<unsigned long long>(offset);
    return s > cut_score || (s == cut_score && o > cut_offset);
  }
};

template <class T, class Pred>
__global__ void FilterCountKernel(CscView<T> x, Pred pred, int64_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t col = warp; col < x.cols; col += warps) {
    Pred p = pred;
    p.Begin(x, col, lane);
    const int64_t start = x.ptr[col];
    const int64_t end = x.ptr[col + 1];
    int64_t count = 0;
    for (int64_t base = start; base < end; base += kWarp) {
      const int64_t at = base + lane;
      const bool keep = at < end && p.Keep(col, at, x.idx[at], x.val[at]);
      count += __popc(__ballot_sync(0xffffffffu, keep));
    }
    if (lane == 0) counts[col] = count;
  }
}

template <class T, class Pred>
__global__ void FilterWriteKernel(CscView<T> x, Pred pred, const int64_t* __restrict__ out_ptr,
                                  int32_t* __restrict__ out_idx, T* __restrict__ out_val) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t col = warp; col < x.cols; col += warps) {
    Pred p = pred;
    p.Begin(x, col, lane);
    const int64_t start = x.ptr[col];
    const int64_t end = x.ptr[col + 1];
    int64_t o = out_ptr[col];
    for (int64_t base = start; base < end; base += kWarp) {
      const int64_t at = base + lane;
      int32_t row = 0;
      T v = T(0);
      bool keep = false;
      if (at < end) {
        row = x.idx[at];
        v = x.val[at];
        keep = p.Keep(col, at, row, v);
      }
      const unsigned mask = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int64_t dst = o + __popc(mask & LaneMaskLt());
        out_idx[dst] = row;
        out_val[dst] = v;
      }
      o += __popc(mask);
    }
  }
}

template <class T, class Pred>
void RunFilter(Ctx& ctx, DevCsc<T>& x, const Pred& pred) {
  const int64_t cols = x.cols;
  prof::Scope scope(ctx.stream, "filter", 0.0);
  ctx.counts.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
  const int threads = 256;
  const int grid = GridFor(cols * kWarp, threads);
  FilterCountKernel<T, Pred><<<grid, threads, 0, ctx.stream>>>(View(x), pred, ctx.counts.data());
  SPAI_LAUNCH_CHECK();
  DevCsc<T> out;
  out.Shape(x.rows, cols, ctx.stream);
  const int64_t nnz = ScanCounts(ctx, ctx.counts.data(), cols, out.ptr.data());
  // algorithmic bytes: x read, the survivors written
  const double entry = static_cast<double>(sizeof(int32_t) + sizeof(T));
  prof::AddBytes("filter", entry * static_cast<double>(x.nnz + (nnz == x.nnz ? 0 : nnz)) +
                               16.0 * static_cast<double>(cols + 1));
  if (nnz == x.nnz) {
    return;  // nothing removed: keep x as it is
  }
  out.ReserveNnz(nnz, ctx.stream);
  FilterWriteKernel<T, Pred><<<grid, threads, 0, ctx.stream>>>(View(x), pred, out.ptr.data(), out.idx.data(),
                                                               out.val.data());
  SPAI_LAUNCH_CHECK();
  x.Swap(out);
}

// ---------------------------------------------------------------------------
// Row scaling / column scaling
template <class T>
__global__ void DiagScaleKernel(const T* __restrict__ d, const int32_t* __restrict__ idx, const T* __restrict__ val,
                                int64_t nnz, T* __restrict__ out) {
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[p] = Mul(d[idx[p]], val[p]);
  }
}

template <class T>
__global__ void ScaleColumnsKernel(CscView<T> x, T* __restrict__ val, const double* __restrict__ scale) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < x.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const T s = static_cast<T>(scale[j]);
    for (int64_t p = x.ptr[j]; p < x.ptr[j + 1]; ++p) val[p] = Mul(val[p], s);
  }
}

// ---------------------------------------------------------------------------
// Padded -> compact columns (warp per column)
template <class T>
__global__ void CompactPaddedKernel(const int64_t* __restrict__ base, const int64_t* __restrict__ base2, int64_t cols,
                                    const int64_t* __restrict__ out_ptr, const int32_t* __restrict__ src_idx,
                                    const T* __restrict__ src_val, int32_t* __restrict__ dst_idx,
                                    T* __restrict__ dst_val, const T* __restrict__ src_val2,
                                    int32_t* __restrict__ dst_idx2, T* __restrict__ dst_val2) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = warp; j < cols; j += warps) {
    const int64_t from = base[j] + (base2 != nullptr ? base2[j] : 0);
    const int64_t to = out_ptr[j];
    const int64_t n = out_ptr[j + 1] - to;
    for (int64_t i = lane; i < n; i += kWarp) {
      const int32_t r = src_idx[from + i];
      if (dst_idx != nullptr) dst_idx[to + i] = r;
      dst_val[to + i] = src_val[from + i];
      if (dst_val2 != nullptr) {
        dst_idx2[to + i] = r;
        dst_val2[to + i] = src_val2[from + i];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// ELL copy
template <class T>
__global__ void EllKernel(CscView<T> x, int width, int32_t* __restrict__ idx, T* __restrict__ val) {
  for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < x.cols;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t start = x.ptr[c];
    const int64_t len = x.ptr[c + 1] - start;
    for (int s = 0; s < width; ++s) {
      const bool in = s < len;
      idx[c * width + s] = in ? x.idx[start + s] : -1;
      if (val != nullptr) val[c * width + s] = in ? x.val[start + s] : T(0);
    }
  }
}

// ---------------------------------------------------------------------------
// Transpose
__global__ void RowCountKernel(const int32_t* __restrict__ idx, int64_t nnz, unsigned long long* __restrict__ counts) {
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    atomicAdd(&counts[idx[p]], 1ull);
  }
}

// Warp per column: every entry takes the next free slot of its row (the order
// inside a row is fixed afterwards by the segment sort).
template <class T>
__global__ void ScatterKernel(CscView<T> x, const int64_t* __restrict__ t_ptr, unsigned int* __restrict__ cursor,
                              int32_t* __restrict__ t_idx, T* __restrict__ t_val) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = warp; j < x.cols; j += warps) {
    for (int64_t p = x.ptr[j] + lane; p < x.ptr[j + 1]; p += kWarp) {
      const int32_t row = x.idx[p];
      const int64_t dst = t_ptr[row] + static_cast<int64_t>(atomicAdd(&cursor[row], 1u));
      t_idx[dst] = static_cast<int32_t>(j);
      t_val[dst] = x.val[p];
    }
  }
}

// Largest value of counts[0, n) into *out (out zeroed by the caller).
__global__ void MaxCountKernel(const int64_t* __restrict__ counts, int64_t n, unsigned long long* __restrict__ out) {
  unsigned long long m = 0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned long long c = static_cast<unsigned long long>(counts[i]);
    m = c > m ? c : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, m, o);
    m = other > m ? other : m;
  }
  if ((threadIdx.x & 31) == 0 && m != 0ull) atomicMax(out, m);
}

// Ascending bitonic sort of 32*R (key, value) pairs, element t*32 + lane in
// register t; keys are distinct except the INT32_MAX padding.
template <int R, class T>
__device__ __forceinline__ void WarpSortPairs(int32_t (&k)[R], T (&v)[R], int lane) {
#pragma unroll
  for (int size = 2; size <= kWarp * R; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= kWarp) {
        const int ts = stride / kWarp;
#pragma unroll
        for (int t = 0; t < R; ++t) {
          const int u = t ^ ts;
          if (u > t) {
            const bool up = ((t * kWarp + lane) & size) == 0;
            if ((k[t] > k[u]) == up) {
              const int32_t kk = k[t];
              k[t] = k[u];
              k[u] = kk;
              const T vv = v[t];
              v[t] = v[u];
              v[u] = vv;
            }
          }
        }
      } else {
#pragma unroll
        for (int t = 0; t < R; ++t) {
          const int32_t ok = __shfl_xor_sync(0xffffffffu, k[t], stride);
          const T ov = __shfl_xor_sync(0xffffffffu, v[t], stride);
          const bool up = ((t * kWarp + lane) & size) == 0;
          const bool lower = (lane & stride) == 0;
          if ((k[t] > ok) == (lower == up)) {
            k[t] = ok;
            v[t] = ov;
          }
        }
      }
    }
  }
}

template <int R, class T>
__device__ __forceinline__ void SortSegmentInRegisters(int64_t start, int len, int32_t* idx, T* val, int lane) {
  int32_t k[R];
  T v[R];
#pragma unroll
  for (int t = 0; t < R; ++t) {
    const int e = t * kWarp + lane;
    k[t] = e < len ? idx[start + e] : INT32_MAX;
    v[t] = e < len ? val[start + e] : T(0);
  }
  WarpSortPairs<R, T>(k, v, lane);
#pragma unroll
  for (int t = 0; t < R; ++t) {
    const int e = t * kWarp + lane;
    if (e < len) {
      idx[start + e] = k[t];
      val[start + e] = v[t];
    }
  }
}

// Warp per segment of at most 256 entries, sorted in registers.
template <class T>
__global__ void SegmentSortRegKernel(const int64_t* __restrict__ ptr, int64_t segments, int32_t* __restrict__ idx,
                                     T* __restrict__ val) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = warp; s < segments; s += warps) {
    const int64_t start = ptr[s];
    const int len = static_cast<int>(ptr[s + 1] - start);
    if (len <= 1 || len > 8 * kWarp) continue;
    if (len <= kWarp) {
      SortSegmentInRegisters<1, T>(start, len, idx, val, lane);
    } else if (len <= 2 * kWarp) {
      SortSegmentInRegisters<2, T>(start, len, idx, val, lane);
    } else if (len <= 4 * kWarp) {
      SortSegmentInRegisters<4, T>(start, len, idx, val, lane);
    } else {
      SortSegmentInRegisters<8, T>(start, len, idx, val, lane);
    }
  }
}

// Bitonic sort of (key, value) pairs in shared memory by one warp or one block.
template <class T>
__device__ void BitonicSortPairs(int32_t* keys, T* vals, int size, int tid, int nthreads, bool block_sync) {
  for (int k = 2; k <= size; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < size; i += nthreads) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const bool ascending = (i & k) == 0;
          const int32_t a = keys[i];
          const int32_t b = keys[ixj];
          if ((a > b) == ascending) {
            keys[i] = b;
            keys[ixj] = a;
            const T tv = vals[i];
            vals[i] = vals[ixj];
            vals[ixj] = tv;
          }
        }
      }
      if (block_sync) {
        __syncthreads();
      } else {
        __syncwarp();
      }
    }
  }
}

constexpr int kWarpSortCap = 512;
constexpr int kBlockSortCap = 8192;

template <class T>
__global__ void SegmentSortWarpKernel(const int64_t* __restrict__ ptr, int64_t segments, int32_t* __restrict__ idx,
                                      T* __restrict__ val) {
  extern __shared__ unsigned char smem_raw[];
  constexpr int kWarpsPerBlock = 4;
  const int warp_in_block = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int32_t* keys = reinterpret_cast<int32_t*>(smem_raw) + warp_in_block * kWarpSortCap;
  T* vals = reinterpret_cast<T*>(smem_raw + kWarpsPerBlock * kWarpSortCap * sizeof(int32_t)) + warp_in_block * kWarpSortCap;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = warp; s < segments; s += warps) {
    const int64_t start = ptr[s];
    const int len = static_cast<int>(ptr[s + 1] - start);
    if (len <= 8 * kWarp || len > kWarpSortCap) continue;
    int size = 1;
    while (size < len) size <<= 1;
    for (int i = lane; i < size; i += kWarp) {
      keys[i] = i < len ? idx[start + i] : INT32_MAX;
      vals[i] = i < len ? val[start + i] : T(0);
    }
    __syncwarp();
    BitonicSortPairs(keys, vals, size, lane, kWarp, false);
    for (int i = lane; i < len; i += kWarp) {
      idx[start + i] = keys[i];
      val[start + i] = vals[i];
    }
    __syncwarp();
  }
}

template <class T>
__global__ void SegmentSortBlockKernel(const int64_t* __restrict__ ptr, int64_t segments, int32_t* __restrict__ idx,
                                       T* __restrict__ val) {
  extern __shared__ unsigned char smem_raw[];
  int32_t* keys = reinterpret_cast<int32_t*>(smem_raw);
  T* vals = reinterpret_cast<T*>(smem_raw + kBlockSortCap * sizeof(int32_t));
  for (int64_t s = blockIdx.x; s < segments; s += gridDim.x) {
    const int64_t start = ptr[s];
    const int len = static_cast<int>(ptr[s + 1] - start);
    if (len <= kWarpSortCap || len > kBlockSortCap) continue;
    int size = 1;
    while (size < len) size <<= 1;
    for (int i = threadIdx.x; i < size; i += blockDim.x) {
      keys[i] = i < len ? idx[start + i] : INT32_MAX;
      vals[i] = i < len ? val[start + i] : T(0);
    }
    __syncthreads();
    BitonicSortPairs(keys, vals, size, threadIdx.x, blockDim.x, true);
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
      idx[start + i] = keys[i];
      val[start + i] = vals[i];
    }
    __syncthreads();
  }
}

// Segments longer than the shared-memory cap (rows of very dense columns):
// chunks of kBlockSortCap entries are sorted in shared memory, then the sorted
// runs are merged in pairs through a scratch copy, pass after pass.  The keys
// of one segment are distinct (the column indices of one row), so an entry's
// place in a merged pair is its place in its own run plus the number of keys
// of the other run below it, found by binary search: every entry moves
// independently.  `starts` / `lens` list the long segments only.
template <class T>
__global__ void LongChunkSortKernel(const int64_t* __restrict__ starts, const int64_t* __restrict__ lens, int64_t count,
                                    int32_t* __restrict__ idx, T* __restrict__ val) {
  extern __shared__ unsigned char smem_raw[];
  int32_t* keys = reinterpret_cast<int32_t*>(smem_raw);
  T* vals = reinterpret_cast<T*>(smem_raw + kBlockSortCap * sizeof(int32_t));
  for (int64_t s = blockIdx.y; s < count; s += gridDim.y) {
    const int64_t len = lens[s];
    for (int64_t c0 = static_cast<int64_t>(blockIdx.x) * kBlockSortCap; c0 < len;
         c0 += static_cast<int64_t>(gridDim.x) * kBlockSortCap) {
      const int64_t start = starts[s] + c0;
      const int n = static_cast<int>(len - c0 < kBlockSortCap ? len - c0 : kBlockSortCap);
      int size = 1;
      while (size < n) size <<= 1;
      for (int i = threadIdx.x; i < size; i += blockDim.x) {
        keys[i] = i < n ? idx[start + i] : INT32_MAX;
        vals[i] = i < n ? val[start + i] : T(0);
      }
      __syncthreads();
      BitonicSortPairs(keys, vals, size, threadIdx.x, blockDim.x, true);
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        idx[start + i] = keys[i];
        val[start + i] = vals[i];
      }
      __syncthreads();
    }
  }
}

// Number of keys in sorted keys[0, n) below key.
__device__ __forceinline__ int64_t CountBelow(const int32_t* keys, int64_t n, int32_t key) {
  int64_t lo = 0;
  int64_t hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < key) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

// One merge pass over runs of `width` entries: src -> dst (same offsets).
template <class T>
__global__ void LongMergeKernel(const int64_t* __restrict__ starts, const int64_t* __restrict__ lens, int64_t count,
                                int64_t width, const int32_t* __restrict__ src_idx, const T* __restrict__ src_val,
                                int32_t* __restrict__ dst_idx, T* __restrict__ dst_val) {
  for (int64_t s = blockIdx.y; s < count; s += gridDim.y) {
    const int64_t start = starts[s];
    const int64_t len = lens[s];
    for (int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < len;
         q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const int64_t pair = q / (2 * width) * (2 * width);
      const int64_t mid = pair + width < len ? pair + width : len;
      const int64_t end = pair + 2 * width < len ? pair + 2 * width : len;
      const int32_t key = src_idx[start + q];
      const int64_t place = q < mid ? (q - pair) + CountBelow(src_idx + start + mid, end - mid, key)
                                    : (q - mid) + CountBelow(src_idx + start + pair, mid - pair, key);
      dst_idx[start + pair + place] = key;
      dst_val[start + pair + place] = src_val[start + q];
    }
  }
}

template <class T>
__global__ void LongCopyKernel(const int64_t* __restrict__ starts, const int64_t* __restrict__ lens, int64_t count,
                               const int32_t* __restrict__ src_idx, const T* __restrict__ src_val,
                               int32_t* __restrict__ dst_idx, T* __restrict__ dst_val) {
  for (int64_t s = blockIdx.y; s < count; s += gridDim.y) {
    for (int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < lens[s];
         q += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      dst_idx[starts[s] + q] = src_idx[starts[s] + q];
      dst_val[starts[s] + q] = src_val[starts[s] + q];
    }
  }
}

template <class T>
void SortLongSegments(Ctx& ctx, const int64_t* ptr, int64_t segments, int32_t* idx, T* val, int64_t longest) {
  // the long segments, listed on the host (this path serves only very dense columns)
  std::vector<int64_t> h_ptr(static_cast<size_t>(segments + 1));
  SPAI_CUDA(cudaMemcpyAsync(h_ptr.data(), ptr, sizeof(int64_t) * (segments + 1), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();
  std::vector<int64_t> list;  // starts, then lengths
  std::vector<int64_t> lengths;
  for (int64_t s = 0; s < segments; ++s) {
    const int64_t len = h_ptr[s + 1] - h_ptr[s];
    if (len > kBlockSortCap) {
      list.push_back(h_ptr[s]);
      lengths.push_back(len);
    }
  }
  const int64_t count = static_cast<int64_t>(list.size());
  if (count == 0) return;
  list.insert(list.end(), lengths.begin(), lengths.end());
  DevBuf<int64_t> table;
  table.Reserve(list.size(), ctx.stream);
  SPAI_CUDA(cudaMemcpyAsync(table.data(), list.data(), sizeof(int64_t) * list.size(), cudaMemcpyHostToDevice,
                            ctx.stream));
  const int64_t* starts = table.data();
  const int64_t* lens = table.data() + count;
  const unsigned grid_y = static_cast<unsigned>(count < 65535 ? count : 65535);
  const size_t block_smem = kBlockSortCap * (sizeof(int32_t) + sizeof(T));
  SPAI_CUDA(cudaFuncSetAttribute(LongChunkSortKernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(block_smem)));
  const unsigned chunks = static_cast<unsigned>((longest + kBlockSortCap - 1) / kBlockSortCap);
  LongChunkSortKernel<T><<<dim3(chunks, grid_y), 1024, block_smem, ctx.stream>>>(starts, lens, count, idx, val);
  SPAI_LAUNCH_CHECK();
  // scratch at the same offsets as the segments
  DevBuf<int32_t> scratch_idx;
  DevBuf<T> scratch_val;
  scratch_idx.Reserve(static_cast<size_t>(h_ptr[segments]), ctx.stream);
  scratch_val.Reserve(static_cast<size_t>(h_ptr[segments]), ctx.stream);
  int32_t* src_idx = idx;
  T* src_val = val;
  int32_t* dst_idx = scratch_idx.data();
  T* dst_val = scratch_val.data();
  const unsigned grid_x = static_cast<unsigned>(std::min<int64_t>((longest + 255) / 256, 4096));
  for (int64_t width = kBlockSortCap; width < longest; width *= 2) {
    LongMergeKernel<T><<<dim3(grid_x, grid_y), 256, 0, ctx.stream>>>(starts, lens, count, width, src_idx, src_val,
                                                                     dst_idx, dst_val);
    SPAI_LAUNCH_CHECK();
    std::swap(src_idx, dst_idx);
    std::swap(src_val, dst_val);
  }
  if (src_idx != idx) {
    LongCopyKernel<T><<<dim3(grid_x, grid_y), 256, 0, ctx.stream>>>(starts, lens, count, src_idx, src_val, idx, val);
    SPAI_LAUNCH_CHECK();
  }
  ctx.Sync();  // the table and the scratch are released on return
}

// Sorts every segment [ptr[s], ptr[s+1]) by index; `longest` bounds the
// segment lengths, so only the kernels that have work are launched.
template <class T>
void SortSegments(Ctx& ctx, const int64_t* ptr, int64_t segments, int32_t* idx, T* val, int64_t longest) {
  if (longest <= 1) return;
  SegmentSortRegKernel<T><<<GridFor(segments * kWarp, 256), 256, 0, ctx.stream>>>(ptr, segments, idx, val);
  SPAI_LAUNCH_CHECK();
  if (longest > 8 * kWarp) {
    const size_t warp_smem = 4 * kWarpSortCap * (sizeof(int32_t) + sizeof(T));
    SegmentSortWarpKernel<T><<<GridFor(segments * kWarp, 128), 128, warp_smem, ctx.stream>>>(ptr, segments, idx, val);
    SPAI_LAUNCH_CHECK();
  }
  if (longest > kWarpSortCap) {
    const size_t block_smem = kBlockSortCap * (sizeof(int32_t) + sizeof(T));
    SPAI_CUDA(cudaFuncSetAttribute(SegmentSortBlockKernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(block_smem)));
    SegmentSortBlockKernel<T><<<GridFor(segments * 1024, 1024), 1024, block_smem, ctx.stream>>>(ptr, segments, idx,
                                                                                               val);
    SPAI_LAUNCH_CHECK();
  }
  if (longest > kBlockSortCap) SortLongSegments(ctx, ptr, segments, idx, val, longest);
}

// ---------------------------------------------------------------------------
// Scores
template <class T>
__global__ void DropScoresKernel(CscView<T> m, const double* __restrict__ cn, const double* __restrict__ tmp,
                                 double* __restrict__ scores) {
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < m.ptr[m.cols];
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = static_cast<double>(m.val[p]);
    const double s = Add(Mul(Mul(v, v), cn[m.idx[p]]), Mul(Mul(2.0, v), tmp[p]));
    scores[p] = isfinite(s) ? s : -INFINITY;
  }
}

template <class T>
__global__ void AbsScoresKernel(const T* __restrict__ val, int64_t nnz, double* __restrict__ scores) {
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    scores[p] = fabs(static_cast<double>(val[p]));
  }
}

// candidate counts per column (entries minus a diagonal)
template <class T>
__global__ void NonDiagonalCountKernel(CscView<T> x, int64_t* __restrict__ counts) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < x.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t c = 0;
    for (int64_t p = x.ptr[j]; p < x.ptr[j + 1]; ++p) c += static_cast<int64_t>(x.idx[p]) != j ? 1 : 0;
    counts[j] = c;
  }
}

// candidate keys in offset order: key[offset] = ordered score bits
template <class T>
__global__ void GatherCandidateKeysKernel(CscView<T> x, const double* __restrict__ scores,
                                          const int64_t* __restrict__ column_base, bool skip_diag,
                                          unsigned long long* __restrict__ keys) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < x.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t o = skip_diag ? column_base[j] : x.ptr[j];
    for (int64_t p = x.ptr[j]; p < x.ptr[j + 1]; ++p) {
      if (skip_diag && static_cast<int64_t>(x.idx[p]) == j) continue;
      keys[o++] = OrderedBits(scores[p]);
    }
  }
}

// Radix select over 128-bit keys (ordered score bits, candidate offset), 8
// bits per pass from the most significant byte.  state = {prefix_hi,
// prefix_lo, remaining rank (1-based)}.
__global__ void RadixHistKernel(const unsigned long long* __restrict__ keys, int64_t count, int pass,
                                const unsigned long long* __restrict__ state, unsigned long long* __restrict__ hist) {
  __shared__ unsigned int local[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) local[i] = 0;
  __syncthreads();
  const unsigned long long prefix_hi = state[0];
  const unsigned long long prefix_lo = state[1];
  for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < count;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const unsigned long long hi = keys[c];
    const unsigned long long lo = static_cast<unsigned long long>(c);
    bool match;
    unsigned digit;
    if (pass < 8) {
      const int shift = 56 - 8 * pass;
      const unsigned long long mask = pass == 0 ? 0ull : (~0ull << (shift + 8));
      match = (hi & mask) == (prefix_hi & mask);
      digit = static_cast<unsigned>((hi >> shift) & 0xFFull);
    } else {
      const int shift = 56 - 8 * (pass - 8);
      const unsigned long long mask = pass == 8 ? 0ull : (~0ull << (shift + 8));
      match = hi == prefix_hi && (lo & mask) == (prefix_lo & mask);
      digit = static_cast<unsigned>((lo >> shift) & 0xFFull);
    }
    if (match) atomicAdd(&local[digit], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    if (local[i] != 0) atomicAdd(&hist[i], static_cast<unsigned long long>(local[i]));
  }
}

__global__ void RadixDecideKernel(int pass, unsigned long long* __restrict__ state, unsigned long long* __restrict__ hist) {
  if (threadIdx.x != 0) return;
  unsigned long long remaining = state[2];
  unsigned long long cumulative = 0;
  int digit = 255;
  for (int b = 0; b < 256; ++b) {
    if (cumulative + hist[b] >= remaining) {
      digit = b;
      break;
    }
    cumulative += hist[b];
  }
  if (pass < 8) {
    state[0] |= static_cast<unsigned long long>(digit) << (56 - 8 * pass);
  } else {
    state[1] |= static_cast<unsigned long long>(digit) << (56 - 8 * (pass - 8));
  }
  state[2] = remaining - cumulative;
  for (int b = 0; b < 256; ++b) hist[b] = 0;
}

template <class S, class D>
__global__ void ConvertKernel(const S* __restrict__ src, D* __restrict__ dst, int64_t n) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    dst[i] = static_cast<D>(src[i]);
  }
}

}  // namespace

// ===========================================================================
int GridFor(int64_t work_items, int threads_per_block) {
  int device = 0;
  cudaGetDevice(&device);
  static int sm_count = 0;
  if (sm_count == 0) {
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
    if (sm_count <= 0) sm_count = 148;
  }
  const int64_t needed = CeilDiv(work_items > 0 ? work_items : 1, threads_per_block);
  const int64_t cap = static_cast<int64_t>(sm_count) * 16;
  return static_cast<int>(needed < cap ? needed : cap);
}

namespace {
struct CachedBlock {
  void* ptr;
  size_t bytes;
};
constexpr size_t kCacheBlocksPerStream = 64;
constexpr size_t kRetiredBlocksPerDevice = 128;
std::mutex g_cache_mutex;
std::map<cudaStream_t, std::vector<CachedBlock>> g_block_cache;
// Blocks of finished contexts (their streams synchronised, so idle), per
// device: any later context on the device takes them before the allocator.
std::map<int, std::vector<CachedBlock>> g_retired;
// the device of every live context stream
std::map<cudaStream_t, int> g_stream_device;

// Index of the smallest block in `blocks` that holds `bytes` without wasting
// more than half of itself, or blocks.size().
size_t BestFit(const std::vector<CachedBlock>& blocks, size_t bytes) {
  size_t best = blocks.size();
  for (size_t i = 0; i < blocks.size(); ++i) {
    const size_t b = blocks[i].bytes;
    if (b >= bytes && b <= 2 * bytes + (size_t{1} << 20) && (best == blocks.size() || b < blocks[best].bytes)) best = i;
  }
  return best;
}

void* TakeAt(std::vector<CachedBlock>& blocks, size_t at, size_t* capacity_bytes) {
  void* p = blocks[at].ptr;
  *capacity_bytes = blocks[at].bytes;
  blocks.erase(blocks.begin() + static_cast<std::ptrdiff_t>(at));
  return p;
}
}  // namespace

void* CacheTake(cudaStream_t stream, size_t bytes, size_t* capacity_bytes) {
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  auto it = g_block_cache.find(stream);
  if (it != g_block_cache.end()) {
    const size_t at = BestFit(it->second, bytes);
    if (at < it->second.size()) return TakeAt(it->second, at, capacity_bytes);
  }
  const auto owner = g_stream_device.find(stream);
  if (owner == g_stream_device.end()) return nullptr;
  auto retired = g_retired.find(owner->second);
  if (retired == g_retired.end()) return nullptr;
  const size_t at = BestFit(retired->second, bytes);
  return at < retired->second.size() ? TakeAt(retired->second, at, capacity_bytes) : nullptr;
}

void CacheGive(cudaStream_t stream, void* block, size_t bytes) {
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  std::vector<CachedBlock>& blocks = g_block_cache[stream];
  blocks.push_back(CachedBlock{block, bytes});
  if (blocks.size() > kCacheBlocksPerStream) {
    // the oldest block goes back to the pool
    cudaFreeAsync(blocks.front().ptr, stream);
    blocks.erase(blocks.begin());
  }
}

void CacheFlush(cudaStream_t stream) {
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  auto it = g_block_cache.find(stream);
  if (it == g_block_cache.end()) return;
  for (const CachedBlock& b : it->second) cudaFreeAsync(b.ptr, stream);
  g_block_cache.erase(it);
}

void CacheRegisterStream(cudaStream_t stream, int device) {
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  g_stream_device[stream] = device;
}

void CacheRetire(cudaStream_t stream, int device) {
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  g_stream_device.erase(stream);
  auto it = g_block_cache.find(stream);
  if (it == g_block_cache.end()) return;
  std::vector<CachedBlock>& retired = g_retired[device];
  for (const CachedBlock& b : it->second) retired.push_back(b);
  g_block_cache.erase(it);
  // keep the newest blocks; the oldest go back to the pool (the stream is idle)
  while (retired.size() > kRetiredBlocksPerDevice) {
    cudaFreeAsync(retired.front().ptr, stream);
    retired.erase(retired.begin());
  }
}

namespace {
// Pinned read-back slots of finished contexts, reused by the next ones
// (cudaMallocHost is slow and cudaFreeHost synchronises the device).
struct PinnedSlots {
  double* scalars;
  int64_t* counts;
  int32_t* flags;
};
std::mutex g_pinned_mutex;
std::vector<PinnedSlots> g_pinned;
}  // namespace

namespace {
// Pinned staging buffers for downloads, reused across calls (pinning memory
// is slow); each call takes one for its duration.
constexpr size_t kStageBytes = size_t{32} << 20;
std::mutex g_stage_mutex;
std::vector<void*> g_stages;

// f(first, last) over [0, n) in up to `parts` contiguous pieces, one thread each.
template <class F>
void HostParallel(int64_t n, int parts, F f) {
  if (parts <= 1 || n < (int64_t{1} << 16)) {
    f(int64_t{0}, n);
    return;
  }
  std::vector<std::thread> pool;
  for (int k = 0; k < parts; ++k) {
    const int64_t first = n * k / parts;
    const int64_t last = n * (k + 1) / parts;
    pool.emplace_back(f, first, last);
  }
  for (auto& t : pool) t.join();
}
}  // namespace

template <class T>
void DownloadWiden(Ctx& ctx, const int32_t* idx_dev, const T* val_dev, int64_t n, int64_t index_offset,
                   int64_t* idx_host, double* val_host) {
  if (n <= 0) return;
  void* stage = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    if (!g_stages.empty()) {
      stage = g_stages.back();
      g_stages.pop_back();
    }
  }
  if (stage == nullptr) SPAI_CUDA(cudaMallocHost(&stage, kStageBytes));
  struct Return {
    void* p;
    ~Return() {
      std::lock_guard<std::mutex> lock(g_stage_mutex);
      g_stages.push_back(p);
    }
  } give_back{stage};
  const int64_t per_chunk = static_cast<int64_t>(kStageBytes / (sizeof(int32_t) + sizeof(T)));
  int32_t* stage_idx = static_cast<int32_t*>(stage);
  T* stage_val = reinterpret_cast<T*>(static_cast<unsigned char*>(stage) + sizeof(int32_t) * per_chunk);
  const int threads = static_cast<int>(std::min(8u, std::max(1u, std::thread::hardware_concurrency())));
  for (int64_t first = 0; first < n; first += per_chunk) {
    const int64_t count = std::min(per_chunk, n - first);
    SPAI_CUDA(cudaMemcpyAsync(stage_idx, idx_dev + first, sizeof(int32_t) * count, cudaMemcpyDeviceToHost, ctx.stream));
    SPAI_CUDA(cudaMemcpyAsync(stage_val, val_dev + first, sizeof(T) * count, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.Sync();
    HostParallel(count, threads, [&](int64_t a, int64_t b) {
      for (int64_t i = a; i < b; ++i) {
        idx_host[first + i] = static_cast<int64_t>(stage_idx[i]) - index_offset;
        val_host[first + i] = static_cast<double>(stage_val[i]);
      }
    });
  }
}

template void DownloadWiden<double>(Ctx&, const int32_t*, const double*, int64_t, int64_t, int64_t*, double*);
template void DownloadWiden<float>(Ctx&, const int32_t*, const float*, int64_t, int64_t, int64_t*, double*);

void Ctx::Init(int device_ordinal) {
  device = device_ordinal;
  SPAI_CUDA(cudaSetDevice(device));
  SPAI_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
  SPAI_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CacheRegisterStream(stream, device);
  cudaMemPool_t pool;
  SPAI_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t threshold = UINT64_MAX;
  SPAI_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  {
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    if (!g_pinned.empty()) {
      host_scalars = g_pinned.back().scalars;
      host_counts = g_pinned.back().counts;
      host_flags = g_pinned.back().flags;
      g_pinned.pop_back();
    }
  }
  if (host_scalars == nullptr) {
    SPAI_CUDA(cudaMallocHost(reinterpret_cast<void**>(&host_scalars), sizeof(double) * kScalarSlots));
    SPAI_CUDA(cudaMallocHost(reinterpret_cast<void**>(&host_counts), sizeof(int64_t) * 8));
    SPAI_CUDA(cudaMallocHost(reinterpret_cast<void**>(&host_flags), sizeof(int32_t) * 8));
  }
  scalars.Reserve(kScalarSlots, stream);
  select_state.Reserve(4, stream);
  histogram.Reserve(256, stream);
  flags.Reserve(8, stream);
  SPAI_CUDA(cudaMemsetAsync(histogram.data(), 0, 256 * sizeof(unsigned long long), stream));
}

void Ctx::Destroy() {
  if (stream != nullptr) {
    cudaStreamSynchronize(stream);
  }
  counts.Release();
  counts2.Release();
  scan_blocks.Release();
  for (auto& p : partials) p.Release();
  tree_scratch.Release();
  scalars.Release();
  for (auto& c : colvec) c.Release();
  select_state.Release();
  histogram.Release();
  flags.Release();
  sg_need.Release();
  sg_counts.Release();
  sg_proj_ptr.Release();
  sg_win_lo.Release();
  sg_win_words.Release();
  sg_cols.Release();
  sg_proj_rows.Release();
  sg_proj_vals.Release();
  sg_fallback.Release();
  sg_maxima.Release();
  sg_ub_ptr.Release();
  sg_bin_cols.Release();
  sg_pad_idx.Release();
  sg_pad_val.Release();
  sg_pad_z.Release();
  pad_idx.Release();
  pad_val.Release();
  if (stream != nullptr) {
    // every block of the stream is idle after the synchronisation above
    CacheRetire(stream, device);
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
    stream = nullptr;
  }
  if (host_scalars != nullptr) {
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    g_pinned.push_back(PinnedSlots{host_scalars, host_counts, host_flags});
  }
  host_scalars = nullptr;
  host_counts = nullptr;
  host_flags = nullptr;
}

void Ctx::Sync() { SPAI_CUDA(cudaStreamSynchronize(stream)); }

void ScanCountsAsync(Ctx& ctx, const int64_t* counts, int64_t n, int64_t* out) {
  if (n <= 0) {
    SPAI_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), ctx.stream));
    return;
  }
  int64_t need = 0;
  for (int64_t m = n; m > 1; m = CeilDiv(m, kScanTile)) need += 2 * CeilDiv(m, kScanTile) + 2;
  ctx.scan_blocks.Reserve(static_cast<size_t>(need + 8), ctx.stream);
  ScanRecursive(ctx, counts, n, out, ctx.scan_blocks, 0);
}

int64_t ScanCounts(Ctx& ctx, const int64_t* counts, int64_t n, int64_t* out) {
  if (n <= 0) {
    SPAI_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), ctx.stream));
    return 0;
  }
  int64_t need = 0;
  for (int64_t m = n; m > 1; m = CeilDiv(m, kScanTile)) need += 2 * CeilDiv(m, kScanTile) + 2;
  ctx.scan_blocks.Reserve(static_cast<size_t>(need + 8), ctx.stream);
  ScanRecursive(ctx, counts, n, out, ctx.scan_blocks, 0);
  SPAI_CUDA(cudaMemcpyAsync(ctx.host_counts, out + n, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();
  return ctx.host_counts[0];
}

void TreeSums(Ctx& ctx, const double* const* partials, int arrays, int64_t n, int slot) {
  TreeDots(ctx, partials, nullptr, arrays, n, slot);
}

void TreeDots(Ctx& ctx, const double* const* x, const double* const* y, int arrays, int64_t n, int slot) {
  if (n <= 0) {
    SPAI_CUDA(cudaMemsetAsync(ctx.scalars.data() + slot, 0, sizeof(double) * arrays, ctx.stream));
    return;
  }
  TreeArgs args{};
  for (int a = 0; a < arrays; ++a) {
    args.src[a] = x[a];
    args.src2[a] = y != nullptr ? y[a] : nullptr;
  }
  int64_t count = n;
  size_t scratch_need = 0;
  for (int64_t m = n; m > kTreeChunk; m = CeilDiv(m, kTreeChunk)) scratch_need += static_cast<size_t>(arrays) * CeilDiv(m, kTreeChunk);
  ctx.tree_scratch.Reserve(scratch_need + 8, ctx.stream);
  size_t scratch_at = 0;
  while (true) {
    const int64_t chunks = CeilDiv(count, kTreeChunk);
    double* dst;
    int64_t stride;
    if (chunks == 1) {
      dst = ctx.scalars.data() + slot;
      stride = 1;
    } else {
      dst = ctx.tree_scratch.data() + scratch_at;
      stride = chunks;
    }
    dim3 grid(static_cast<unsigned>(chunks), static_cast<unsigned>(arrays));
    TreeChunkKernel<<<grid, kTreeLanes, 0, ctx.stream>>>(args, count, dst, stride);
    SPAI_LAUNCH_CHECK();
    if (chunks == 1) break;
    for (int a = 0; a < arrays; ++a) {
      args.src[a] = dst + a * chunks;
      args.src2[a] = nullptr;
    }
    scratch_at += static_cast<size_t>(arrays) * chunks;
    count = chunks;
  }
}

void SegmentTree::Build(Ctx& ctx, const std::vector<int64_t>& offsets) {
  const int64_t segments = static_cast<int64_t>(offsets.size()) - 1;
  segments_ = segments;
  final_at_.assign(static_cast<size_t>(segments), -1);
  levels_.clear();
  std::vector<int64_t> table;
  // the segments still being reduced: [lo, hi) in the current level's source
  std::vector<int64_t> lo(offsets.begin(), offsets.end() - 1);
  std::vector<int64_t> hi(offsets.begin() + 1, offsets.end());
  std::vector<int64_t> owner(static_cast<size_t>(segments));
  for (int64_t s = 0; s < segments; ++s) owner[s] = s;
  int64_t slots = 0;
  while (!owner.empty()) {
    std::vector<int64_t> start;
    std::vector<int64_t> end;
    std::vector<int64_t> dst;
    std::vector<int64_t> next_lo;
    std::vector<int64_t> next_hi;
    std::vector<int64_t> next_owner;
    for (size_t k = 0; k < owner.size(); ++k) {
      const int64_t len = hi[k] - lo[k];
      if (len <= 0) continue;  // an empty segment sums to +0.0, as TreeSums gives
      const int64_t chunks = CeilDiv(len, kTreeChunk);
      if (chunks == 1) final_at_[owner[k]] = slots;
      for (int64_t c = 0; c < chunks; ++c) {
        start.push_back(lo[k] + c * kTreeChunk);
        end.push_back(std::min(lo[k] + (c + 1) * kTreeChunk, hi[k]));
        dst.push_back(slots + c);
      }
      if (chunks > 1) {
        next_lo.push_back(slots);
        next_hi.push_back(slots + chunks);
        next_owner.push_back(owner[k]);
      }
      slots += chunks;
    }
    if (!start.empty()) {
      Level level;
      level.blocks = static_cast<int64_t>(start.size());
      level.table_at = static_cast<int64_t>(table.size());
      table.insert(table.end(), start.begin(), start.end());
      table.insert(table.end(), end.begin(), end.end());
      table.insert(table.end(), dst.begin(), dst.end());
      levels_.push_back(level);
    }
    lo.swap(next_lo);
    hi.swap(next_hi);
    owner.swap(next_owner);
  }
  slots_ = slots;
  table_.Reserve(table.empty() ? 1 : table.size(), ctx.stream);
  if (!table.empty()) {
    SPAI_CUDA(cudaMemcpyAsync(table_.data(), table.data(), sizeof(int64_t) * table.size(), cudaMemcpyHostToDevice,
                              ctx.stream));
  }
  ctx.Sync();
}

void SegmentTree::Sums(Ctx& ctx, const double* const* partials, int arrays, double* out) {
  if (arrays > 8) throw std::invalid_argument("SegmentTree::Sums takes at most 8 arrays");
  values_.Reserve(static_cast<size_t>(arrays) * (slots_ > 0 ? slots_ : 1), ctx.stream);
  TreeArgs args{};
  for (size_t l = 0; l < levels_.size(); ++l) {
    for (int a = 0; a < arrays; ++a) args.src[a] = l == 0 ? partials[a] : values_.data() + a * slots_;
    dim3 grid(static_cast<unsigned>(levels_[l].blocks), static_cast<unsigned>(arrays));
    SegmentChunkKernel<<<grid, kTreeLanes, 0, ctx.stream>>>(args, table_.data() + levels_[l].table_at,
                                                            levels_[l].blocks, values_.data(), slots_);
    SPAI_LAUNCH_CHECK();
  }
  host_.resize(static_cast<size_t>(arrays) * slots_);
  if (slots_ > 0) {
    SPAI_CUDA(cudaMemcpyAsync(host_.data(), values_.data(), sizeof(double) * host_.size(), cudaMemcpyDeviceToHost,
                              ctx.stream));
  }
  ctx.Sync();
  for (int a = 0; a < arrays; ++a) {
    for (int64_t s = 0; s < segments_; ++s) {
      const int64_t at = final_at_[s];
      out[a * segments_ + s] = at < 0 ? 0.0 : host_[a * slots_ + at];
    }
  }
}

void FetchScalars(Ctx& ctx, int first_slot, int count, double* out) {
  SPAI_CUDA(cudaMemcpyAsync(ctx.host_scalars, ctx.scalars.data() + first_slot, sizeof(double) * count,
                            cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();
  std::memcpy(out, ctx.host_scalars, sizeof(double) * count);
}

template <class T>
void ColumnSquares(Ctx& ctx, CscView<T> x, double* partial) {
  ColumnSquaresKernel<T><<<GridFor(x.cols, 128), 128, 0, ctx.stream>>>(x, partial);
  SPAI_LAUNCH_CHECK();
}

template <class T>
void ColumnDots(Ctx& ctx, CscView<T> x, CscView<T> y, double* partial) {
  ColumnDotsKernel<T><<<GridFor(x.cols, 128), 128, 0, ctx.stream>>>(x, y, partial);
  SPAI_LAUNCH_CHECK();
}

template <class T>
void Union(Ctx& ctx, const DevCsc<T>& y, bool scale_y, double ys, const DevCsc<T>& x, double xs, DevCsc<T>& out,
           UnionMode mode) {
  const int64_t cols = y.cols;
  ctx.counts.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
  const int grid = GridFor(cols, 128);
  const int64_t cap = UnionWarpCap();
  const bool half_sum = mode == UnionMode::kHalfSum;
  prof::Scope scope(ctx.stream, "union", 0.0);
  // algorithmic bytes: both operands read, the union written
  auto account = [&](const DevCsc<T>& u) {
    const double entry = static_cast<double>(sizeof(int32_t) + sizeof(T));
    prof::AddBytes("union", entry * static_cast<double>(y.nnz + x.nnz + u.nnz) + 24.0 * static_cast<double>(cols + 1));
  };
  {
    DevCsc<T> single;
    if (UnionPadded(ctx, y, scale_y, ys, x, xs, half_sum, !half_sum, single)) {
      account(single);
      out.Swap(single);
      return;
    }
  }
  UnionCountWarp(ctx, y, x, ctx.counts.data());
  UnionKernel<T, false><<<grid, 128, 0, ctx.stream>>>(View(y), View(x), scale_y, ys, xs, static_cast<int>(mode), cap,
                                                      ctx.counts.data(), nullptr, nullptr, nullptr);
  SPAI_LAUNCH_CHECK();
  DevCsc<T> result;
  result.Shape(y.rows, cols, ctx.stream);
  const int64_t nnz = ScanCounts(ctx, ctx.counts.data(), cols, result.ptr.data());
  result.ReserveNnz(nnz, ctx.stream);
  SPAI_CUDA(cudaMemsetAsync(ctx.flags.data(), 0, sizeof(int32_t), ctx.stream));
  UnionWriteWarp(ctx, y, x, scale_y, ys, xs, half_sum, !half_sum, result, ctx.flags.data());
  UnionKernel<T, true><<<grid, 128, 0, ctx.stream>>>(View(y), View(x), scale_y, ys, xs, static_cast<int>(mode), cap,
                                                     nullptr, result.ptr.data(), result.idx.data(), result.val.data());
  SPAI_LAUNCH_CHECK();
  if (!half_sum) {
    // exact zeros from y + a*x (rare): remove them like Eigen's prune(0.0)
    SPAI_CUDA(cudaMemcpyAsync(ctx.host_flags, ctx.flags.data(), sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.Sync();
    if (ctx.host_flags[0] != 0) DropZeros(ctx, result);
  }
  account(result);
  out.Swap(result);
}

template <class T>
void DiagScale(Ctx& ctx, const T* d, const DevCsc<T>& b, DevCsc<T>& out, bool prune_zeros) {
  DevCsc<T> result;
  result.Shape(b.rows, b.cols, ctx.stream);
  result.ReserveNnz(b.nnz, ctx.stream);
  SPAI_CUDA(cudaMemcpyAsync(result.ptr.data(), b.ptr.data(), sizeof(int64_t) * (b.cols + 1), cudaMemcpyDeviceToDevice,
                            ctx.stream));
  if (b.nnz > 0) {
    SPAI_CUDA(cudaMemcpyAsync(result.idx.data(), b.idx.data(), sizeof(int32_t) * b.nnz, cudaMemcpyDeviceToDevice,
                              ctx.stream));
    DiagScaleKernel<T><<<GridFor(b.nnz, 256), 256, 0, ctx.stream>>>(d, b.idx.data(), b.val.data(), b.nnz,
                                                                   result.val.data());
    SPAI_LAUNCH_CHECK();
  }
  out.Swap(result);
  if (prune_zeros) DropZeros(ctx, out);
}

template <class T>
void ScaleColumns(Ctx& ctx, DevCsc<T>& x, const double* scale) {
  ScaleColumnsKernel<T><<<GridFor(x.cols, 128), 128, 0, ctx.stream>>>(View(x), x.val.data(), scale);
  SPAI_LAUNCH_CHECK();
  DropZeros(ctx, x);
}

template <class T>
void CompactPadded(Ctx& ctx, const int64_t* base, const int64_t* base2, int64_t cols, const int64_t* out_ptr,
                   const int32_t* src_idx, const T* src_val, int32_t* dst_idx, T* dst_val) {
  CompactPaddedKernel<T><<<GridFor(cols * kWarp, 256), 256, 0, ctx.stream>>>(base, base2, cols, out_ptr, src_idx,
                                                                            src_val, dst_idx, dst_val, nullptr,
                                                                            nullptr, nullptr);
  SPAI_LAUNCH_CHECK();
}

template <class T>
void CompactPaddedPair(Ctx& ctx, const int64_t* base, int64_t cols, const int64_t* out_ptr, const int32_t* src_idx,
                       const T* src_val, int32_t* dst_idx, T* dst_val, const T* src_val2, int32_t* dst_idx2,
                       T* dst_val2) {
  CompactPaddedKernel<T><<<GridFor(cols * kWarp, 256), 256, 0, ctx.stream>>>(base, nullptr, cols, out_ptr, src_idx,
                                                                            src_val, dst_idx, dst_val, src_val2,
                                                                            dst_idx2, dst_val2);
  SPAI_LAUNCH_CHECK();
}

template <class T>
void BuildEll(Ctx& ctx, const DevCsc<T>& x, int width, int32_t* idx, T* val) {
  EllKernel<T><<<GridFor(x.cols, 128), 128, 0, ctx.stream>>>(View(x), width, idx, val);
  SPAI_LAUNCH_CHECK();
}

template <class T>
void DropZeros(Ctx& ctx, DevCsc<T>& x) {
  RunFilter(ctx, x, KeepNonZero<T>{});
}

template <class T>
void PruneColumnRelative(Ctx& ctx, DevCsc<T>& m) {
  RunFilter(ctx, m, KeepColumnRelative<T>{});
}

template <class T>
void PruneAbsAtMost(Ctx& ctx, DevCsc<T>& x, double limit) {
  RunFilter(ctx, x, KeepAboveLimit<T>{limit});
}

template <class T>
void PruneAbsAtMostPerColumn(Ctx& ctx, DevCsc<T>& x, const double* column_limit) {
  RunFilter(ctx, x, KeepAboveLimit<T>{0.0, column_limit});
}

template <class T>
void KeepTopKPerColumn(Ctx& ctx, DevCsc<T>& x, int64_t k, bool protect_diagonal) {
  KeepTopK<T> pred;
  pred.k = k;
  pred.protect = protect_diagonal;
  RunFilter(ctx, x, pred);
}

template <class T>
void GlobalDropByScore(Ctx& ctx, DevCsc<T>& x, const double* entry_scores, bool skip_diagonal, int64_t drop) {
  const int64_t cols = x.cols;
  ctx.counts2.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
  int64_t candidates = x.nnz;
  const int64_t* column_base = nullptr;
  if (skip_diagonal) {
    ctx.counts.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
    NonDiagonalCountKernel<T><<<GridFor(cols, 128), 128, 0, ctx.stream>>>(View(x), ctx.counts.data());
    SPAI_LAUNCH_CHECK();
    candidates = ScanCounts(ctx, ctx.counts.data(), cols, ctx.counts2.data());
    column_base = ctx.counts2.data();
  }
  if (drop <= 0 || drop > candidates) {
    throw std::invalid_argument("Invalid global sparse dropping count");
  }
  DevBuf<unsigned long long> keys;
  keys.Reserve(static_cast<size_t>(candidates), ctx.stream);
  GatherCandidateKeysKernel<T><<<GridFor(cols, 128), 128, 0, ctx.stream>>>(View(x), entry_scores, column_base,
                                                                          skip_diagonal, keys.data());
  SPAI_LAUNCH_CHECK();
  unsigned long long init[3] = {0ull, 0ull, static_cast<unsigned long long>(drop)};
  SPAI_CUDA(cudaMemcpyAsync(ctx.select_state.data(), init, sizeof(init), cudaMemcpyHostToDevice, ctx.stream));
  SPAI_CUDA(cudaMemsetAsync(ctx.histogram.data(), 0, 256 * sizeof(unsigned long long), ctx.stream));
  const int grid = GridFor(candidates, 256);
  for (int pass = 0; pass < 16; ++pass) {
    RadixHistKernel<<<grid, 256, 0, ctx.stream>>>(keys.data(), candidates, pass, ctx.select_state.data(),
                                                  ctx.histogram.data());
    SPAI_LAUNCH_CHECK();
    RadixDecideKernel<<<1, 32, 0, ctx.stream>>>(pass, ctx.select_state.data(), ctx.histogram.data());
    SPAI_LAUNCH_CHECK();
  }
  KeepAboveCutoff<T> pred;
  pred.scores = entry_scores;
  pred.column_base = column_base;
  pred.cutoff = ctx.select_state.data();
  pred.skip_diag = skip_diagonal;
  RunFilter(ctx, x, pred);
  keys.Release();
}

template <class T>
void Transpose(Ctx& ctx, const DevCsc<T>& x, DevCsc<T>& t) {
  prof::Scope scope(ctx.stream, "transpose", 0.0);
  DevCsc<T> result;
  result.Shape(x.cols, x.rows, ctx.stream);
  ctx.counts.Reserve(static_cast<size_t>(x.rows + 1), ctx.stream);
  unsigned long long* row_counts = reinterpret_cast<unsigned long long*>(ctx.counts.data());
  SPAI_CUDA(cudaMemsetAsync(row_counts, 0, sizeof(int64_t) * (x.rows + 1), ctx.stream));
  if (x.nnz > 0) {
    RowCountKernel<<<GridFor(x.nnz, 256), 256, 0, ctx.stream>>>(x.idx.data(), x.nnz, row_counts);
    SPAI_LAUNCH_CHECK();
  }
  // the longest row, read back by the scan's synchronisation
  unsigned long long* longest = ctx.select_state.data() + 3;
  SPAI_CUDA(cudaMemsetAsync(longest, 0, sizeof(unsigned long long), ctx.stream));
  MaxCountKernel<<<GridFor(x.rows, 256), 256, 0, ctx.stream>>>(ctx.counts.data(), x.rows, longest);
  SPAI_LAUNCH_CHECK();
  SPAI_CUDA(cudaMemcpyAsync(ctx.host_counts + 1, longest, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx.stream));
  const int64_t nnz = ScanCounts(ctx, ctx.counts.data(), x.rows, result.ptr.data());
  const int64_t longest_row = ctx.host_counts[1];
  result.ReserveNnz(nnz, ctx.stream);
  unsigned int* cursor = reinterpret_cast<unsigned int*>(row_counts);
  SPAI_CUDA(cudaMemsetAsync(cursor, 0, sizeof(unsigned int) * x.rows, ctx.stream));
  if (nnz > 0) {
    ScatterKernel<T><<<GridFor(x.cols * kWarp, 256), 256, 0, ctx.stream>>>(View(x), result.ptr.data(), cursor,
                                                                          result.idx.data(), result.val.data());
    SPAI_LAUNCH_CHECK();
    SortSegments<T>(ctx, result.ptr.data(), x.rows, result.idx.data(), result.val.data(), longest_row);
  }
  // algorithmic bytes: x read, its transpose written
  prof::AddBytes("transpose", static_cast<double>(sizeof(int32_t) + sizeof(T)) * 2.0 * static_cast<double>(x.nnz) +
                                  8.0 * static_cast<double>(x.cols + 1 + x.rows + 1));
  t.Swap(result);
}

template <class T>
void Copy(Ctx& ctx, const DevCsc<T>& x, DevCsc<T>& out) {
  DevCsc<T> result;
  result.Shape(x.rows, x.cols, ctx.stream);
  result.ReserveNnz(x.nnz, ctx.stream);
  SPAI_CUDA(cudaMemcpyAsync(result.ptr.data(), x.ptr.data(), sizeof(int64_t) * (x.cols + 1), cudaMemcpyDeviceToDevice,
                            ctx.stream));
  if (x.nnz > 0) {
    SPAI_CUDA(cudaMemcpyAsync(result.idx.data(), x.idx.data(), sizeof(int32_t) * x.nnz, cudaMemcpyDeviceToDevice,
                              ctx.stream));
    SPAI_CUDA(cudaMemcpyAsync(result.val.data(), x.val.data(), sizeof(T) * x.nnz, cudaMemcpyDeviceToDevice,
                              ctx.stream));
  }
  out.Swap(result);
}

template <class T>
void DropScores(Ctx& ctx, const DevCsc<T>& m, const double* col_norm2, const double* tmp, double* scores) {
  if (m.nnz == 0) return;
  DropScoresKernel<T><<<GridFor(m.nnz, 256), 256, 0, ctx.stream>>>(View(m), col_norm2, tmp, scores);
  SPAI_LAUNCH_CHECK();
}

template <class T>
void AbsScores(Ctx& ctx, const DevCsc<T>& x, double* scores) {
  if (x.nnz == 0) return;
  AbsScoresKernel<T><<<GridFor(x.nnz, 256), 256, 0, ctx.stream>>>(x.val.data(), x.nnz, scores);
  SPAI_LAUNCH_CHECK();
}

void FillZero(Ctx& ctx, int64_t* ptr, int64_t n) {
  SPAI_CUDA(cudaMemsetAsync(ptr, 0, sizeof(int64_t) * n, ctx.stream));
}

template <class S, class D>
void ConvertValues(Ctx& ctx, const S* src, D* dst, int64_t n) {
  if (n <= 0) return;
  ConvertKernel<S, D><<<GridFor(n, 256), 256, 0, ctx.stream>>>(src, dst, n);
  SPAI_LAUNCH_CHECK();
}

#define SPAI_INSTANTIATE(T)                                                                                   \
  template void ColumnSquares<T>(Ctx&, CscView<T>, double*);                                                  \
  template void ColumnDots<T>(Ctx&, CscView<T>, CscView<T>, double*);                                         \
  template void Union<T>(Ctx&, const DevCsc<T>&, bool, double, const DevCsc<T>&, double, DevCsc<T>&, UnionMode); \
  template void DiagScale<T>(Ctx&, const T*, const DevCsc<T>&, DevCsc<T>&, bool);                             \
  template void ScaleColumns<T>(Ctx&, DevCsc<T>&, const double*);                                             \
  template void DropZeros<T>(Ctx&, DevCsc<T>&);                                                               \
  template void BuildEll<T>(Ctx&, const DevCsc<T>&, int, int32_t*, T*);                                         \
  template void CompactPaddedPair<T>(Ctx&, const int64_t*, int64_t, const int64_t*, const int32_t*, const T*,         \
                                     int32_t*, T*, const T*, int32_t*, T*);                                      \
  template void CompactPadded<T>(Ctx&, const int64_t*, const int64_t*, int64_t, const int64_t*, const int32_t*,      \
                                 const T*, int32_t*, T*);                                                        \
  template void PruneColumnRelative<T>(Ctx&, DevCsc<T>&);                                                     \
  template void PruneAbsAtMost<T>(Ctx&, DevCsc<T>&, double);                                                  \
  template void PruneAbsAtMostPerColumn<T>(Ctx&, DevCsc<T>&, const double*);                                  \
  template void KeepTopKPerColumn<T>(Ctx&, DevCsc<T>&, int64_t, bool);                                        \
  template void GlobalDropByScore<T>(Ctx&, DevCsc<T>&, const double*, bool, int64_t);                         \
  template void Transpose<T>(Ctx&, const DevCsc<T>&, DevCsc<T>&);                                             \
  template void Copy<T>(Ctx&, const DevCsc<T>&, DevCsc<T>&);                                                  \
  template void DropScores<T>(Ctx&, const DevCsc<T>&, const double*, const double*, double*);                 \
  template void AbsScores<T>(Ctx&, const DevCsc<T>&, double*);

SPAI_INSTANTIATE(double)
SPAI_INSTANTIATE(float)

template void ConvertValues<double, float>(Ctx&, const double*, float*, int64_t);
template void ConvertValues<float, double>(Ctx&, const float*, double*, int64_t);
template void ConvertValues<double, double>(Ctx&, const double*, double*, int64_t);

}  // namespace spai
