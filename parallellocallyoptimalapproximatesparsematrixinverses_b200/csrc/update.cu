// Column-merging updates of M on sm_100a, one warp per column.
//
// Union (out = ys*Y (+) xs*X, or 0.5*(Y + X)): every lane takes entries of
// both input columns and computes its output slot directly -- an entry of Y
// lands at (#Y before it) + (#X rows below it that Y lacks), an entry of X
// found nowhere in Y at (#unmatched X before it) + (#Y rows below it) -- from
// binary searches into the other column and a per-column prefix of the
// matched X entries kept in shared memory.  No serial merge, no sort.
//
// SymmetrizeAndDrop fuses the drop step of the global methods
// (dropping.cpp:106-135, plus the optional per-column top-k): the merged
// column of 0.5*(M + M^T) is built in shared memory, its 2-norm is summed in
// row order by one lane (the reference's per-column sequential sum), the
// relative threshold is applied there, the top-k rule by a bitonic sort of
// (|v|, position) keys in registers, and the survivors are written once, at
// an upper-bound offset, then compacted.  This replaces transpose-union,
// threshold-filter and top-k-filter passes over HBM.

#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"
#include "ops.cuh"
#include "profile.cuh"
#include "select.cuh"

namespace spai {

namespace {

constexpr int kUnionWarpCap = 1024;  // longest X column the warp union takes (shared-memory prefix)

// First position in idx[lo, hi) whose row is >= key.
__device__ __forceinline__ int64_t LowerBound(const int32_t* idx, int64_t lo, int64_t hi, int32_t key) {
  while (lo < hi) {
    const int64_t mid = lo + ((hi - lo) >> 1);
    if (idx[mid] < key) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

// Values of one merged entry, in the arithmetic of the thread-per-column
// union: the storage type's (FP64 for double, FP32 for float storage).
template <class T>
__device__ __forceinline__ T Both(T y, T x, bool scale_y, T ys, T xs, bool half_sum) {
  if (half_sum) return Mul(T(0.5), Add(y, x));
  return Add(scale_y ? Mul(ys, y) : y, Mul(xs, x));
}

template <class T>
__device__ __forceinline__ T LeftOnly(T y, bool scale_y, T ys, bool half_sum) {
  if (half_sum) return Mul(T(0.5), Add(y, T(0)));
  return Add(scale_y ? Mul(ys, y) : y, T(0));
}

template <class T>
__device__ __forceinline__ T RightOnly(T x, T xs, bool half_sum) {
  if (half_sum) return Mul(T(0.5), Add(T(0), x));
  return Add(T(0), Mul(xs, x));
}

// Number of rows of X(:, j) also present in Y(:, j) (warp-uniform).
template <class T>
__device__ int64_t CommonRows(const CscView<T>& y, const CscView<T>& x, int64_t j, int lane) {
  const int64_t ys = y.ptr[j];
  const int64_t ye = y.ptr[j + 1];
  const int64_t xs = x.ptr[j];
  const int64_t xe = x.ptr[j + 1];
  int64_t matched = 0;
  for (int64_t base = xs; base < xe; base += kWarp) {
    const int64_t q = base + lane;
    bool hit = false;
    if (q < xe) {
      const int32_t row = x.idx[q];
      const int64_t r = LowerBound(y.idx, ys, ye, row);
      hit = r < ye && y.idx[r] == row;
    }
    matched += __popc(__ballot_sync(0xffffffffu, hit));
  }
  return matched;
}

// mx_prefix[i] = number of the first i entries of X(:, j) whose row is in
// Y(:, j), for i = 0..nx.  Ends with __syncwarp.
template <class T>
__device__ void MatchedPrefix(const CscView<T>& y, const CscView<T>& x, int64_t j, int* mx_prefix, int lane) {
  const int64_t ys = y.ptr[j];
  const int64_t ye = y.ptr[j + 1];
  const int64_t xs = x.ptr[j];
  const int64_t xe = x.ptr[j + 1];
  int running = 0;
  for (int64_t base = xs; base < xe; base += kWarp) {
    const int64_t q = base + lane;
    bool hit = false;
    if (q < xe) {
      const int32_t row = x.idx[q];
      const int64_t r = LowerBound(y.idx, ys, ye, row);
      hit = r < ye && y.idx[r] == row;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, hit);
    if (q < xe) mx_prefix[q - xs] = running + __popc(mask & LaneMaskBelow());
    running += __popc(mask);
  }
  if (lane == 0) mx_prefix[xe - xs] = running;
  __syncwarp();
}

// Calls emit(rank, row, value) for every entry of the merged column j; rank
// is the entry's position in the merged, row-sorted column.
template <class T, class Emit>
__device__ void MergeColumn(const CscView<T>& y, const CscView<T>& x, int64_t j, bool scale_y, double ys_scale,
                            double xs_scale, bool half_sum, const int* mx_prefix, int lane, Emit emit) {
  const int64_t ys = y.ptr[j];
  const int64_t ye = y.ptr[j + 1];
  const int64_t xs = x.ptr[j];
  const int64_t xe = x.ptr[j + 1];
  for (int64_t p = ys + lane; p < ye; p += kWarp) {
    const int32_t row = y.idx[p];
    const int64_t r = LowerBound(x.idx, xs, xe, row);
    const int64_t rank = (p - ys) + (r - xs) - mx_prefix[r - xs];
    const T ysc = static_cast<T>(ys_scale);
    const T xsc = static_cast<T>(xs_scale);
    const T v = (r < xe && x.idx[r] == row) ? Both(y.val[p], x.val[r], scale_y, ysc, xsc, half_sum)
                                            : LeftOnly(y.val[p], scale_y, ysc, half_sum);
    emit(rank, row, v);
  }
  for (int64_t q = xs + lane; q < xe; q += kWarp) {
    const int32_t row = x.idx[q];
    const int64_t r = LowerBound(y.idx, ys, ye, row);
    if (r < ye && y.idx[r] == row) continue;
    const int64_t qq = q - xs;
    const int64_t rank = qq - mx_prefix[qq] + (r - ys);
    emit(rank, row, RightOnly(x.val[q], static_cast<T>(xs_scale), half_sum));
  }
}

template <class T>
__global__ void UnionCountWarpKernel(CscView<T> y, CscView<T> x, int64_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = warp; j < y.cols; j += warps) {
    const int64_t nx = x.ptr[j + 1] - x.ptr[j];
    if (nx > kUnionWarpCap) continue;  // the thread-per-column kernel takes it
    const int64_t ny = y.ptr[j + 1] - y.ptr[j];
    const int64_t matched = CommonRows(y, x, j, lane);
    if (lane == 0) counts[j] = ny + nx - matched;
  }
}

template <class T>
__global__ void UnionWriteWarpKernel(CscView<T> y, CscView<T> x, bool scale_y, double ys, double xs, bool half_sum,
                                     bool prune, const int64_t* __restrict__ out_ptr, int32_t* __restrict__ out_idx,
                                     T* __restrict__ out_val, int32_t* __restrict__ flag) {
  extern __shared__ int union_smem[];
  const int lane = threadIdx.x & 31;
  int* mx_prefix = union_smem + (threadIdx.x >> 5) * (kUnionWarpCap + 1);
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  bool zero_seen = false;
  for (int64_t j = warp; j < y.cols; j += warps) {
    const int64_t nx = x.ptr[j + 1] - x.ptr[j];
    if (nx > kUnionWarpCap) continue;
    MatchedPrefix(y, x, j, mx_prefix, lane);
    const int64_t base = out_ptr[j];
    MergeColumn(y, x, j, scale_y, ys, xs, half_sum, mx_prefix, lane, [&](int64_t rank, int32_t row, T stored) {
      out_idx[base + rank] = row;
      out_val[base + rank] = stored;
      if (prune && stored == T(0)) zero_seen = true;
    });
    __syncwarp();
  }
  if (__any_sync(0xffffffffu, zero_seen) && lane == 0) atomicOr(flag, 1);
}

// MatchedPrefix and MergeColumn over row keys staged in shared memory
// (yk, xk: the two columns' rows; pre: nx + 1 ints); values are read from
// the input columns.  Emits nothing and returns the merged length when it
// exceeds `cap`.
template <class T, class Emit>
__device__ int MergeShared(const CscView<T>& y, const CscView<T>& x, int64_t j, int32_t* yk, int32_t* xk, int* pre,
                           bool scale_y, double ys_scale, double xs_scale, bool half_sum, int cap, int lane,
                           Emit emit) {
  const int64_t ys = y.ptr[j];
  const int64_t xs = x.ptr[j];
  const int ny = static_cast<int>(y.ptr[j + 1] - ys);
  const int nx = static_cast<int>(x.ptr[j + 1] - xs);
  for (int i = lane; i < ny; i += kWarp) yk[i] = y.idx[ys + i];
  for (int i = lane; i < nx; i += kWarp) xk[i] = x.idx[xs + i];
  __syncwarp();
  int running = 0;
  for (int base = 0; base < nx; base += kWarp) {
    const int q = base + lane;
    bool hit = false;
    if (q < nx) {
      const int32_t row = xk[q];
      const int r = LowerBoundShared(yk, ny, row);
      hit = r < ny && yk[r] == row;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, hit);
    if (q < nx) pre[q] = running + __popc(mask & LaneMaskBelow());
    running += __popc(mask);
  }
  if (lane == 0) pre[nx] = running;
  __syncwarp();
  const int merged = ny + nx - running;
  if (merged > cap) return merged;
  const T ysc = static_cast<T>(ys_scale);
  const T xsc = static_cast<T>(xs_scale);
  for (int p = lane; p < ny; p += kWarp) {
    const int32_t row = yk[p];
    const int r = LowerBoundShared(xk, nx, row);
    const T yv = y.val[ys + p];
    const T v = (r < nx && xk[r] == row) ? Both(yv, x.val[xs + r], scale_y, ysc, xsc, half_sum)
                                         : LeftOnly(yv, scale_y, ysc, half_sum);
    emit(p + r - pre[r], row, v);
  }
  for (int q = lane; q < nx; q += kWarp) {
    const int32_t row = xk[q];
    const int r = LowerBoundShared(yk, ny, row);
    if (r < ny && yk[r] == row) continue;
    emit(q - pre[q] + r, row, RightOnly(x.val[xs + q], xsc, half_sum));
  }
  return merged;
}

constexpr int kUnionPadCap = 256;  // longest input column of the single-pass union (keeps 8 blocks resident)

// Single-pass union: column j of the result goes to out at y.ptr[j] +
// x.ptr[j] (an upper bound of its offset); exact zeros are pruned in place
// (kAxpby) and counts[j] is the surviving length.  Columns with an input
// longer than kUnionPadCap set `overflow` (the caller then uses the
// two-pass kernels).
template <class T>
__global__ void UnionPaddedKernel(CscView<T> y, CscView<T> x, bool scale_y, double ys_scale, double xs_scale,
                                  bool half_sum, bool prune, int64_t* __restrict__ counts,
                                  int32_t* __restrict__ out_idx, T* __restrict__ out_val,
                                  int32_t* __restrict__ overflow) {
  extern __shared__ __align__(16) int32_t union_pad_smem[];
  const int lane = threadIdx.x & 31;
  int32_t* yk = union_pad_smem + (threadIdx.x >> 5) * (3 * kUnionPadCap + 4);
  int32_t* xk = yk + kUnionPadCap;
  int* pre = xk + kUnionPadCap;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = warp; j < y.cols; j += warps) {
    const int64_t ny = y.ptr[j + 1] - y.ptr[j];
    const int64_t nx = x.ptr[j + 1] - x.ptr[j];
    if (ny > kUnionPadCap || nx > kUnionPadCap) {
      if (lane == 0) atomicOr(overflow, 1);
      continue;
    }
    const int64_t base = y.ptr[j] + x.ptr[j];
    bool zero = false;
    const int merged = MergeShared(y, x, j, yk, xk, pre, scale_y, ys_scale, xs_scale, half_sum, 2 * kUnionPadCap,
                                   lane, [&](int rank, int32_t row, T stored) {
                                     out_idx[base + rank] = row;
                                     out_val[base + rank] = stored;
                                     if (prune && stored == T(0)) zero = true;
                                   });
    int kept = merged;
    if (__any_sync(0xffffffffu, zero)) {
      // rare: squeeze the exact zeros out of this column, in order
      __syncwarp();
      int64_t at = base;
      for (int i0 = 0; i0 < merged; i0 += kWarp) {
        const int i = i0 + lane;
        int32_t r = 0;
        T v = T(0);
        if (i < merged) {
          r = out_idx[base + i];
          v = out_val[base + i];
        }
        const bool keep = i < merged && !(v == T(0));
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        __syncwarp();
        if (keep) {
          out_idx[at + __popc(mask & LaneMaskBelow())] = r;
          out_val[at + __popc(mask & LaneMaskBelow())] = v;
        }
        at += __popc(mask);
        __syncwarp();
      }
      kept = static_cast<int>(at - base);
    }
    if (lane == 0) counts[j] = kept;
    __syncwarp();
  }
}

// One pass: survivors of column j go to out at ub_ptr[j] = m.ptr[j] (+
// mt.ptr[j] when symmetric), their number to counts[j]; `overflow` is set
// when a column exceeds kDropCap (the caller then discards the pass).
template <class T>
__global__ void __launch_bounds__(256, 4) SymmetrizeDropKernel(CscView<T> m, CscView<T> mt, bool symmetric, int64_t topk,
                                     int64_t* __restrict__ counts, int32_t* __restrict__ out_idx,
                                     T* __restrict__ out_val, int32_t* __restrict__ overflow) {
  extern __shared__ __align__(16) unsigned char drop_smem[];
  const int lane = threadIdx.x & 31;
  DropSlab s = SlabFor(drop_smem + (threadIdx.x >> 5) * DropSlabBytes());
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t j = warp; j < m.cols; j += warps) {
    const int64_t ny = m.ptr[j + 1] - m.ptr[j];
    int count;
    if (symmetric) {
      const int64_t nx = mt.ptr[j + 1] - mt.ptr[j];
      if (nx > kDropCap || ny > kDropCap) {
        if (lane == 0) atomicOr(overflow, 1);
        continue;
      }
      const int merged = MergeShared(m, mt, j, s.yk, s.xk, s.mx_prefix, false, 1.0, 1.0, true, kDropCap, lane,
                                     [&](int rank, int32_t row, T v) {
        s.keys[rank] = row;
        s.vals[rank] = static_cast<double>(v);  // the value M would store
      });
      if (merged > kDropCap) {
        if (lane == 0) atomicOr(overflow, 1);
        __syncwarp();
        continue;
      }
      count = merged;
    } else {
      if (ny > kDropCap) {
        if (lane == 0) atomicOr(overflow, 1);
        continue;
      }
      count = static_cast<int>(ny);
      const int64_t base = m.ptr[j];
      for (int i = lane; i < count; i += kWarp) {
        s.keys[i] = m.idx[base + i];
        s.vals[i] = static_cast<double>(m.val[base + i]);
      }
    }
    __syncwarp();
    const int kept = DecideDrops(s, count, j, topk, lane);
    int64_t out = m.ptr[j] + (symmetric ? mt.ptr[j] : 0);
    for (int base = 0; base < count; base += kWarp) {
      const int i = base + lane;
      const bool keep = i < count && s.keep[i] != 0;
      const unsigned mask = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int64_t o = out + __popc(mask & LaneMaskBelow());
        out_idx[o] = s.keys[i];
        out_val[o] = static_cast<T>(s.vals[i]);
      }
      out += __popc(mask);
    }
    if (lane == 0) counts[j] = kept;
    __syncwarp();
  }
}

}  // namespace

int UnionWarpCap() { return kUnionWarpCap; }

template <class T>
void UnionCountWarp(Ctx& ctx, const DevCsc<T>& y, const DevCsc<T>& x, int64_t* counts) {
  UnionCountWarpKernel<T><<<GridFor(y.cols * kWarp, 256), 256, 0, ctx.stream>>>(View(y), View(x), counts);
  SPAI_LAUNCH_CHECK();
}

template <class T>
void UnionWriteWarp(Ctx& ctx, const DevCsc<T>& y, const DevCsc<T>& x, bool scale_y, double ys, double xs, bool half_sum,
                    bool prune, DevCsc<T>& out, int32_t* flag) {
  constexpr int kWarps = 8;
  const size_t smem = static_cast<size_t>(kWarps) * (kUnionWarpCap + 1) * sizeof(int);
  UnionWriteWarpKernel<T><<<GridFor(y.cols * kWarp, kWarps * kWarp), kWarps * kWarp, smem, ctx.stream>>>(
      View(y), View(x), scale_y, ys, xs, half_sum, prune, out.ptr.data(), out.idx.data(), out.val.data(), flag);
  SPAI_LAUNCH_CHECK();
}

template <class T>
bool UnionPadded(Ctx& ctx, const DevCsc<T>& y, bool scale_y, double ys, const DevCsc<T>& x, double xs, bool half_sum,
                 bool prune, DevCsc<T>& out) {
  const int64_t cols = y.cols;
  const int64_t padded = y.nnz + x.nnz;
  const size_t slots = static_cast<size_t>(padded > 0 ? padded : 1);
  ctx.pad_idx.Reserve(slots, ctx.stream);
  ctx.pad_val.Reserve(slots * sizeof(T), ctx.stream);
  int32_t* tmp_idx = ctx.pad_idx.data();
  T* tmp_val = reinterpret_cast<T*>(ctx.pad_val.data());
  ctx.counts.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
  int32_t* overflow = ctx.flags.data() + 2;
  SPAI_CUDA(cudaMemsetAsync(overflow, 0, sizeof(int32_t), ctx.stream));
  constexpr int kWarps = 8;
  const size_t smem = static_cast<size_t>(kWarps) * (3 * kUnionPadCap + 4) * sizeof(int32_t);
  SPAI_CUDA(cudaFuncSetAttribute(UnionPaddedKernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
  const int grid = GridFor(cols * kWarp, kWarps * kWarp);
  UnionPaddedKernel<T><<<grid, kWarps * kWarp, smem, ctx.stream>>>(View(y), View(x), scale_y, ys, xs, half_sum, prune,
                                                                   ctx.counts.data(), tmp_idx, tmp_val, overflow);
  SPAI_LAUNCH_CHECK();
  SPAI_CUDA(cudaMemcpyAsync(ctx.host_flags + 2, overflow, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
  out.Shape(y.rows, cols, ctx.stream);
  const int64_t nnz = ScanCounts(ctx, ctx.counts.data(), cols, out.ptr.data());  // synchronises: flag is read
  if (ctx.host_flags[2] != 0) return false;
  out.ReserveNnz(nnz, ctx.stream);
  CompactPadded(ctx, y.ptr.data(), x.ptr.data(), cols, out.ptr.data(), tmp_idx, tmp_val, out.idx.data(),
                out.val.data());
  return true;
}

template <class T>
bool SymmetrizeAndDrop(Ctx& ctx, DevCsc<T>& m, bool symmetric, int64_t topk) {
  prof::Scope scope(ctx.stream, "drop_update", 0.0);
  const int64_t cols = m.cols;
  DevCsc<T> mt;
  if (symmetric) Transpose(ctx, m, mt);
  const CscView<T> mt_view = symmetric ? View(mt) : View(m);
  constexpr int kWarps = 8;
  const size_t smem = DropSlabBytes() * kWarps;
  SPAI_CUDA(cudaFuncSetAttribute(SymmetrizeDropKernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
  const int grid = GridFor(cols * kWarp, kWarps * kWarp);
  // survivors land at m.ptr[j] (+ mt.ptr[j]): an upper bound of column j's merged length
  const int64_t padded = m.nnz + (symmetric ? mt.nnz : 0);
  const size_t slots = static_cast<size_t>(padded > 0 ? padded : 1);
  ctx.pad_idx.Reserve(slots, ctx.stream);
  ctx.pad_val.Reserve(slots * sizeof(T), ctx.stream);
  int32_t* tmp_idx = ctx.pad_idx.data();
  T* tmp_val = reinterpret_cast<T*>(ctx.pad_val.data());
  ctx.counts.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
  int32_t* overflow = ctx.flags.data() + 1;
  SPAI_CUDA(cudaMemsetAsync(overflow, 0, sizeof(int32_t), ctx.stream));
  SymmetrizeDropKernel<T><<<grid, kWarps * kWarp, smem, ctx.stream>>>(View(m), mt_view, symmetric, topk,
                                                                      ctx.counts.data(), tmp_idx, tmp_val, overflow);
  SPAI_LAUNCH_CHECK();
  SPAI_CUDA(cudaMemcpyAsync(ctx.host_flags + 1, overflow, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
  DevCsc<T> out;
  out.Shape(m.rows, cols, ctx.stream);
  const int64_t nnz = ScanCounts(ctx, ctx.counts.data(), cols, out.ptr.data());  // synchronises: flag is read
  if (ctx.host_flags[1] != 0) return false;
  out.ReserveNnz(nnz, ctx.stream);
  CompactPadded(ctx, m.ptr.data(), symmetric ? mt.ptr.data() : nullptr, cols, out.ptr.data(), tmp_idx, tmp_val,
                out.idx.data(), out.val.data());
  // algorithmic bytes: M and M^T read (and M^T formed: M read, M^T written), the result written
  const double entry = static_cast<double>(sizeof(int32_t) + sizeof(T));
  const double ptrs = 8.0 * static_cast<double>(cols + 1);
  const double mt_nnz = symmetric ? static_cast<double>(mt.nnz) : 0.0;
  prof::AddBytes("drop_update", entry * (static_cast<double>(m.nnz) + 3.0 * mt_nnz + static_cast<double>(nnz)) +
                                    ptrs * (symmetric ? 4.0 : 2.0));
  m.Swap(out);
  return true;
}

template void UnionCountWarp<double>(Ctx&, const DevCsc<double>&, const DevCsc<double>&, int64_t*);
template void UnionCountWarp<float>(Ctx&, const DevCsc<float>&, const DevCsc<float>&, int64_t*);
template void UnionWriteWarp<double>(Ctx&, const DevCsc<double>&, const DevCsc<double>&, bool, double, double, bool,
                                     bool, DevCsc<double>&, int32_t*);
template void UnionWriteWarp<float>(Ctx&, const DevCsc<float>&, const DevCsc<float>&, bool, double, double, bool, bool,
                                    DevCsc<float>&, int32_t*);
template bool UnionPadded<double>(Ctx&, const DevCsc<double>&, bool, double, const DevCsc<double>&, double, bool,
                                  bool, DevCsc<double>&);
template bool UnionPadded<float>(Ctx&, const DevCsc<float>&, bool, double, const DevCsc<float>&, double, bool, bool,
                                 DevCsc<float>&);
template bool SymmetrizeAndDrop<double>(Ctx&, DevCsc<double>&, bool, int64_t);
template bool SymmetrizeAndDrop<float>(Ctx&, DevCsc<float>&, bool, int64_t);

}  // namespace spai
