#pragma once
// Host-callable device operations on sparse matrices in HBM.  Each operation
// is stream-ordered on Ctx::stream.  Functions that must size an output read
// one int64 back from the device (ScanCounts); everything else is
// asynchronous.

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device.cuh"

namespace spai {

// Per-call device context: stream, scratch buffers and pinned readback slots.
struct Ctx {
  cudaStream_t stream = nullptr;
  int device = 0;
  int sm_count = 148;
  DevBuf<int64_t> counts;       // per-column counts, n + 1
  DevBuf<int64_t> counts2;      // second per-column count array
  DevBuf<int64_t> scan_blocks;  // scan tile sums
  DevBuf<double> partials[8];   // per-column partial sums of the canonical reductions
  DevBuf<double> tree_scratch;  // tree-sum chunk sums
  DevBuf<double> scalars;       // device-resident reduction results (kScalarSlots)
  DevBuf<double> colvec[6];     // per-column coefficient vectors (inner-outer)
  DevBuf<unsigned long long> select_state;  // radix-select state
  DevBuf<unsigned long long> histogram;     // radix-select histogram
  DevBuf<int32_t> flags;        // device flags (zero pruning happened, overflow)
  // SpGEMM per-call scratch, kept so the iteration loop reaches the allocator only on growth
  DevBuf<int64_t> sg_need;
  DevBuf<int64_t> sg_counts;
  DevBuf<int64_t> sg_proj_ptr;
  DevBuf<int32_t> sg_win_lo;
  DevBuf<int32_t> sg_win_words;
  DevBuf<int32_t> sg_cols;
  DevBuf<int32_t> sg_proj_rows;
  DevBuf<unsigned char> sg_proj_vals;
  DevBuf<unsigned char> sg_fallback;
  DevBuf<unsigned long long> sg_maxima;
  DevBuf<int64_t> sg_ub_ptr;             // padded column offsets (scan of the upper bounds)
  DevBuf<int32_t> sg_bin_cols;           // column lists of the SpGEMM window bins
  DevBuf<int32_t> sg_pad_idx;            // padded output rows
  DevBuf<unsigned char> sg_pad_val;      // padded output values
  DevBuf<unsigned char> sg_pad_z;        // padded fused Z values
  DevBuf<int32_t> pad_idx;               // padded rows of the union and drop steps
  DevBuf<unsigned char> pad_val;         // padded values of the union and drop steps
  double* host_scalars = nullptr;   // pinned, kScalarSlots
  int64_t* host_counts = nullptr;   // pinned, 8
  int32_t* host_flags = nullptr;    // pinned, 8

  static constexpr int kScalarSlots = 64;

  void Init(int device_ordinal);
  void Destroy();
  void Sync();
  double* Partial(int i, int64_t n) {
    partials[i].Reserve(static_cast<size_t>(n), stream);
    return partials[i].data();
  }
};

// out[0] = 0, out[i + 1] = counts[0] + ... + counts[i]; returns out[n] (one
// device-to-host read).  counts and out must not alias.
int64_t ScanCounts(Ctx& ctx, const int64_t* counts, int64_t n, int64_t* out);
// The same scan without the read-back (stream-ordered, no synchronisation).
void ScanCountsAsync(Ctx& ctx, const int64_t* counts, int64_t n, int64_t* out);

// Moves column j of a padded matrix -- out_ptr[j+1] - out_ptr[j] entries
// starting at base[j] (+ base2[j] when base2 is given) of src -- to
// out_ptr[j] of dst.  dst_idx may be null (values only).
// Two padded matrices of one pattern (rows in src_idx) in one pass: a matrix
// and a second value array, e.g. R and Z = Pr*R.
template <class T>
void CompactPaddedPair(Ctx& ctx, const int64_t* base, int64_t cols, const int64_t* out_ptr, const int32_t* src_idx,
                       const T* src_val, int32_t* dst_idx, T* dst_val, const T* src_val2, int32_t* dst_idx2,
                       T* dst_val2);
template <class T>
void CompactPadded(Ctx& ctx, const int64_t* base, const int64_t* base2, int64_t cols, const int64_t* out_ptr,
                   const int32_t* src_idx, const T* src_val, int32_t* dst_idx, T* dst_val);

// Canonical reduction: the fixed 4096-wide tree over `n` partial sums.
// Results land in ctx.scalars[slot + i] for i < arrays; read them with
// FetchScalars.
void TreeSums(Ctx& ctx, const double* const* partials, int arrays, int64_t n, int slot);
// Same tree over the products x[a][i] * y[a][i] (dot products of vectors).
void TreeDots(Ctx& ctx, const double* const* x, const double* const* y, int arrays, int64_t n, int slot);
void FetchScalars(Ctx& ctx, int first_slot, int count, double* out);

// The same tree applied to every segment [offsets[s], offsets[s + 1]) of a
// per-column array on its own (the diagonal blocks of a batch): each
// segment's sum has the bits TreeSums gives for that segment alone.  Build
// once per segmentation; every Sums call is one launch per tree level over
// all segments and one read-back.
class SegmentTree {
 public:
  void Build(Ctx& ctx, const std::vector<int64_t>& offsets);
  // out[a * segments + s] = the tree sum of partials[a] over segment s (host), a < arrays <= 8.
  void Sums(Ctx& ctx, const double* const* partials, int arrays, double* out);
  int64_t segments() const { return segments_; }

 private:
  struct Level {
    int64_t blocks = 0;
    int64_t table_at = 0;
  };
  std::vector<Level> levels_;
  std::vector<int64_t> final_at_;  // slot of each segment's sum (-1: empty segment)
  int64_t segments_ = 0;
  int64_t slots_ = 0;              // per-array slots over all levels
  DevBuf<int64_t> table_;
  DevBuf<double> values_;
  std::vector<double> host_;
};

// Host copies of a device index array (int32, minus index_offset, widened to
// int64) and value array (T, widened to double), n entries each, through a
// pinned staging buffer reused across calls and widened by several host
// threads.  Synchronises the stream.
template <class T>
void DownloadWiden(Ctx& ctx, const int32_t* idx_dev, const T* val_dev, int64_t n, int64_t index_offset,
                   int64_t* idx_host, double* val_host);

// Per-column sequential partial sums (storage order, as Eigen within a column).
template <class T>
void ColumnSquares(Ctx& ctx, CscView<T> x, double* partial);
// sum over rows present in both columns of x*y, ascending rows.
template <class T>
void ColumnDots(Ctx& ctx, CscView<T> x, CscView<T> y, double* partial);

// Union combination: out = ys*Y (+) xs*X (sparse_operations.cpp:22-49).
// kAxpby prunes exact zeros; kHalfSum computes 0.5*(y + x) and keeps zeros
// (the symmetrisation of dropping.cpp:115-117).
enum class UnionMode { kAxpby = 0, kHalfSum = 1 };
template <class T>
void Union(Ctx& ctx, const DevCsc<T>& y, bool scale_y, double ys, const DevCsc<T>& x, double xs, DevCsc<T>& out,
           UnionMode mode);

// Fused drop step of M (dropping.cpp:106-135 and the per-column top-k rule):
// M := 0.5 (M + M^T) when symmetric, relative threshold prune, then at most
// topk entries per column (topk == 0: no cap).  Returns false, leaving M
// untouched, when a column is too long for the shared-memory kernel.
template <class T>
bool SymmetrizeAndDrop(Ctx& ctx, DevCsc<T>& m, bool symmetric, int64_t topk);

// Warp-per-column union kernels (update.cu), used by Union().
template <class T>
void UnionCountWarp(Ctx& ctx, const DevCsc<T>& y, const DevCsc<T>& x, int64_t* counts);
template <class T>
void UnionWriteWarp(Ctx& ctx, const DevCsc<T>& y, const DevCsc<T>& x, bool scale_y, double ys, double xs, bool half_sum,
                    bool prune, DevCsc<T>& out, int32_t* flag);
int UnionWarpCap();
// Single-pass union into `out` (fresh); false when a column is too long for
// it (then nothing is written and the two-pass kernels must run).
template <class T>
bool UnionPadded(Ctx& ctx, const DevCsc<T>& y, bool scale_y, double ys, const DevCsc<T>& x, double xs, bool half_sum,
                 bool prune, DevCsc<T>& out);

// Fixed-width (ELL) copy of x: slot s of column c is entry s of x(:, c), or
// index -1 (value 0) past the column's end; width >= the longest column.
// val may be null (indices only).
template <class T>
void BuildEll(Ctx& ctx, const DevCsc<T>& x, int width, int32_t* idx, T* val);

// Row scaling out = diag(d) * b (Pr * X with a diagonal Pr); optional zero pruning.
template <class T>
void DiagScale(Ctx& ctx, const T* d, const DevCsc<T>& b, DevCsc<T>& out, bool prune_zeros);

// x(:, j) *= scale[j] (device array), then exact zeros pruned (sparse_operations.cpp:28-39).
template <class T>
void ScaleColumns(Ctx& ctx, DevCsc<T>& x, const double* scale);

// Filters (each writes a compacted copy and swaps it in).
template <class T>
void DropZeros(Ctx& ctx, DevCsc<T>& x);
// keep iff v != 0 and (diagonal or |v| >= eps * ||column||_2)   (dropping.cpp:124-133)
template <class T>
void PruneColumnRelative(Ctx& ctx, DevCsc<T>& m);
// keep iff !(|v| <= limit)   (dropping.cpp:182-185 with limit = ||X||_F * eps)
template <class T>
void PruneAbsAtMost(Ctx& ctx, DevCsc<T>& x, double limit);
// the same with a limit per column (device array of x.cols values)
template <class T>
void PruneAbsAtMostPerColumn(Ctx& ctx, DevCsc<T>& x, const double* column_limit);
// keep the k largest (|v|, row) per column; the diagonal is always kept (and
// counts toward k) when protect_diagonal.
template <class T>
void KeepTopKPerColumn(Ctx& ctx, DevCsc<T>& x, int64_t k, bool protect_diagonal);

// Global budget selection (dropping.cpp:64-93,145-171,192-222).
// scores: one key per candidate, candidates enumerated in column-major order
// (for M the diagonal is excluded); drops the `drop` smallest (score, offset).
template <class T>
void GlobalDropByScore(Ctx& ctx, DevCsc<T>& x, const double* entry_scores, bool skip_diagonal, int64_t drop);

// Transpose with rows sorted inside every output column.
template <class T>
void Transpose(Ctx& ctx, const DevCsc<T>& x, DevCsc<T>& t);

// Copies.
template <class T>
void Copy(Ctx& ctx, const DevCsc<T>& x, DevCsc<T>& out);

// Residual-aware drop score for every entry of M (dropping.cpp:19-29):
// s = v*v*cn[row] + 2*v*tmp, non-finite -> -inf; tmp aligned with M entries.
template <class T>
void DropScores(Ctx& ctx, const DevCsc<T>& m, const double* col_norm2, const double* tmp, double* scores);

// |v| for every entry (direction budget key).
template <class T>
void AbsScores(Ctx& ctx, const DevCsc<T>& x, double* scores);

// Number of structural nonzeros (host value already known) -- helper to set
// every column pointer of an empty matrix.
void FillZero(Ctx& ctx, int64_t* ptr, int64_t n);

// Convert values between storage precisions (identical pattern).
template <class S, class D>
void ConvertValues(Ctx& ctx, const S* src, D* dst, int64_t n);

}  // namespace spai
