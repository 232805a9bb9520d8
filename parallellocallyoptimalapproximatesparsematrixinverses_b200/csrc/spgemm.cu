// SpGEMM C = X * B on sm_100a in four stages.
//
//  1. row-set count   (one warp per output column) -- the distinct rows of the
//     union of X(:,k), k in B(:,j):
//       bitmap: candidates set bits of a shared-memory bitmap over the row
//               window (all candidate rows within 65,536 rows: every stencil
//               operator); popcounts give the count;
//       hash:   otherwise an open-addressing hash in shared memory (global
//               memory beyond the largest bin).
//  2. row-set list    (same warps, after the scan of the counts) -- writes the
//     sorted rows of every column (bitmap: lane-blocked popcount prefix;
//     hash: compaction + bitonic sort) and the column id of every entry.
//  3. values          (one thread per output entry) -- entry (i, j) walks row
//     i of X (CSR copy) in ascending k, finds each k in column j of B by a
//     binary search (eight searches in flight per thread), and accumulates
//     the first product x*y then += x*y in ascending k: the reference's
//     accumulation order (Eigen's conservative sparse product), no FMA.
//     Products and sums use the storage type's arithmetic: FP64 for double
//     storage (bit-compatible with the reference), FP32 multiply and
//     accumulate for float storage (the mixed-precision form); the global
//     reductions built from them are FP64 either way.
//  4. column sums     (one thread per column) -- sequential per-column sums in
//     row order for the global reductions (||R||^2, the MR projection).
//
// Stages 1-2 are latency-bound warp-per-column work on small shared-memory
// structures; stage 3, where the arithmetic happens, is parallel over all
// output entries so the memory system sees enough independent loads.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include "device.cuh"
#include "ops.cuh"
#include "profile.cuh"
#include "colkit.cuh"
#include "spgemm.cuh"

namespace spai {

namespace {

constexpr int kBitmapMaxWords = 2048;  // 65,536-row window
// window-word bins of the bitmap row-set kernels
constexpr int kWordBins[] = {128, 512, 1040, kBitmapMaxWords};
constexpr int kWordBinCount = 4;
// maxima[] layout: 0 max upper bound, 1 max nnz(B col), 4.. bitmap bin populations, 8 hash columns
constexpr int kMaxUb = 0;
constexpr int kMaxNb = 1;
constexpr int kPopulation = 4;
constexpr int kHashColumns = 8;
constexpr int kSumUb = 9;
constexpr int kMaximaSlots = 16;


__device__ __forceinline__ uint32_t Slot(int32_t key, int bits) {
  return (static_cast<uint32_t>(key) * 2654435761u) >> (32 - bits);
}



// Returns true when `key` was not in the table yet.
__device__ __forceinline__ bool InsertKey(int32_t* table, int bits, int32_t key) {
  const uint32_t mask = (1u << bits) - 1u;
  uint32_t h = Slot(key, bits);
  while (true) {
    const int32_t old = atomicCAS(&table[h], kEmpty, key);
    if (old == kEmpty) return true;
    if (old == key) return false;
    h = (h + 1u) & mask;
  }
}



// Calls f(row) for every candidate row of output column `col`, the rows of
// X(:,k) for k in B(:,col) flattened across the 32 lanes; f returns true for
// a new row.  Returns the warp-uniform number of new rows.
template <class T, class F>
__device__ int ForEachCandidate(const CscView<T>& x, const CscView<T>& b, int64_t col, int32_t* prefix,
                                int64_t* xstart, int lane, F f) {
  int added = 0;
  const int64_t start = b.ptr[col];
  const int64_t end = b.ptr[col + 1];
  for (int64_t base = start; base < end; base += kWarp) {
    const int64_t p = base + lane;
    int64_t xs = 0;
    int len = 0;
    if (p < end) {
      const int32_t k = b.idx[p];
      xs = x.ptr[k];
      len = static_cast<int>(x.ptr[k + 1] - xs);
    }
    int inclusive = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, inclusive, o);
      if (lane >= o) inclusive += y;
    }
    const int total = __shfl_sync(0xffffffffu, inclusive, 31);
    prefix[lane] = inclusive - len;
    xstart[lane] = xs;
    __syncwarp();
    for (int e0 = 0; e0 < total; e0 += kWarp) {
      const int e = e0 + lane;
      bool fresh = false;
      if (e < total) {
        int lo = 0;
        int hi = 31;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (prefix[mid] <= e) {
            lo = mid;
          } else {
            hi = mid - 1;
          }
        }
        fresh = f(x.idx[xstart[lo] + (e - prefix[lo])]);
      }
      added += __popc(__ballot_sync(0xffffffffu, fresh));
    }
    __syncwarp();
  }
  return added;
}

// Per-lane variant for narrow windows: lane l walks the X columns of B
// entries l, l+32, ...; the B indices and X column bounds of up to four
// rounds are loaded before any row, so the loads overlap.
template <class T, class F>
__device__ inline void ForEachCandidateByLane(const CscView<T>& x, const CscView<T>& b, int64_t col, int lane, F f) {
  constexpr int kRounds = 4;
  const int64_t start = b.ptr[col];
  const int64_t end = b.ptr[col + 1];
  for (int64_t base = start; base < end; base += kRounds * kWarp) {
    int32_t k[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      const int64_t p = base + lane + r * kWarp;
      k[r] = p < end ? b.idx[p] : -1;
    }
    int64_t xs[kRounds];
    int64_t xe[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      xs[r] = k[r] >= 0 ? x.ptr[k[r]] : 0;
      xe[r] = k[r] >= 0 ? x.ptr[k[r] + 1] : 0;
    }
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      for (int64_t q0 = xs[r]; q0 < xe[r]; q0 += 8) {
        int32_t rows[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) rows[u] = q0 + u < xe[r] ? x.idx[q0 + u] : -1;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          if (rows[u] >= 0) f(rows[u]);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Stages 1-2: row sets
template <class T>
struct RowSetArgs {
  CscView<T> x;
  CscView<T> b;
  const int64_t* need;       // hash path: table slots needed (2 * upper bound)
  const int32_t* win_lo;     // first row of the candidate window
  const int32_t* win_words;  // window length in 32-row words (0: no candidates)
  bool add_diag;
  bool list;                 // false: count rows; true: write them
  int64_t* counts;           // count mode output
  const int64_t* c_ptr;      // list mode: output offsets
  int32_t* rows;             // list mode: sorted rows
  int32_t* cols;             // list mode: column id of every entry
  unsigned char* global_space;
};

__host__ __device__ inline size_t BitmapBytes(int words) { return Round16(static_cast<size_t>(words) * 4); }

template <class T>
__global__ void BitmapRowSetKernel(RowSetArgs<T> a, int words_cap, int lo_words, int hi_words) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  uint32_t* bm = reinterpret_cast<uint32_t*>(smem + warp_in_block * BitmapBytes(words_cap));
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t col = warp; col < a.b.cols; col += warps) {
    const int words = a.win_words[col];
    if (words <= lo_words || words > hi_words) continue;
    const int32_t lo = a.win_lo[col];
    ClearWords(bm, words, lane);
    __syncwarp();
    if (a.add_diag && lane == 0) {
      const int off = static_cast<int>(col) - lo;
      atomicOr(&bm[off >> 5], 1u << (off & 31));
    }
    ForEachCandidateByLane(a.x, a.b, col, lane, [&](int32_t row) {
      const int off = row - lo;
      atomicOr(&bm[off >> 5], 1u << (off & 31));
    });
    __syncwarp();
    if (!a.list) {
      int count = 0;
      for (int w = lane; w < words; w += kWarp) count += __popc(bm[w]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
      if (lane == 0) a.counts[col] = count;
    } else {
      // lane-blocked prefix over the window words, then each lane writes its rows in order
      const int per_lane = (words + kWarp - 1) / kWarp;
      const int w0 = lane * per_lane;
      const int w1 = min(w0 + per_lane, words);
      int local = 0;
      for (int w = w0; w < w1; ++w) local += __popc(bm[w]);
      int inclusive = local;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inclusive, o);
        if (lane >= o) inclusive += y;
      }
      int64_t out = a.c_ptr[col] + (inclusive - local);
      const int32_t col32 = static_cast<int32_t>(col);
      for (int w = w0; w < w1; ++w) {
        uint32_t bits = bm[w];
        while (bits != 0u) {
          const int bit = __ffs(bits) - 1;
          a.rows[out] = lo + (w << 5) + bit;
          a.cols[out] = col32;
          ++out;
          bits &= bits - 1u;
        }
      }
    }
    __syncwarp();
  }
}

__host__ __device__ inline size_t HashRowSetBytes(int slots) {
  // keys + sorted (half) + flattening scratch
  return Round16(static_cast<size_t>(slots) * 4) + Round16(static_cast<size_t>(slots) * 2) +
         Round16(32 * sizeof(int64_t)) + Round16(33 * 4);
}

template <class T>
__global__ void HashRowSetKernel(RowSetArgs<T> a, int slots, int64_t lo_need, int64_t hi_need) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int warps_per_block = blockDim.x >> 5;
  const size_t bytes = HashRowSetBytes(slots);
  unsigned char* base = a.global_space != nullptr
                            ? a.global_space + (static_cast<size_t>(blockIdx.x) * warps_per_block + warp_in_block) * bytes
                            : smem + warp_in_block * bytes;
  int32_t* keys = reinterpret_cast<int32_t*>(base);
  int32_t* sorted = reinterpret_cast<int32_t*>(base + Round16(static_cast<size_t>(slots) * 4));
  int64_t* xstart = reinterpret_cast<int64_t*>(base + Round16(static_cast<size_t>(slots) * 4) +
                                               Round16(static_cast<size_t>(slots) * 2));
  int32_t* prefix = reinterpret_cast<int32_t*>(reinterpret_cast<unsigned char*>(xstart) + Round16(32 * sizeof(int64_t)));
  const int bits = Log2(slots);
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t col = warp; col < a.b.cols; col += warps) {
    if (a.win_words[col] <= kBitmapMaxWords) continue;
    const int64_t need = a.need[col];
    if (need <= lo_need || need > hi_need) continue;
    ClearTable(keys, slots, lane);
    __syncwarp();
    int count = 0;
    if (a.add_diag) {
      bool fresh = false;
      if (lane == 0) fresh = InsertKey(keys, bits, static_cast<int32_t>(col));
      count += __popc(__ballot_sync(0xffffffffu, fresh));
    }
    count += ForEachCandidate(a.x, a.b, col, prefix, xstart, lane,
                              [&](int32_t row) { return InsertKey(keys, bits, row); });
    __syncwarp();
    if (!a.list) {
      if (lane == 0) a.counts[col] = count;
      __syncwarp();
      continue;
    }
    int n = 0;
    for (int s = 0; s < slots; s += kWarp) {
      const int32_t key = keys[s + lane];
      const bool occupied = key != kEmpty;
      const unsigned mask = __ballot_sync(0xffffffffu, occupied);
      if (occupied) sorted[n + __popc(mask & LaneMaskBelow())] = key;
      n += __popc(mask);
    }
    int size = 1;
    while (size < n) size <<= 1;
    for (int i = n + lane; i < size; i += kWarp) sorted[i] = INT32_MAX;
    __syncwarp();
    for (int k = 2; k <= size; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = lane; i < size; i += kWarp) {
          const int ixj = i ^ j;
          if (ixj > i) {
            const int32_t u = sorted[i];
            const int32_t v = sorted[ixj];
            if ((u > v) == ((i & k) == 0)) {
              sorted[i] = v;
              sorted[ixj] = u;
            }
          }
        }
        __syncwarp();
      }
    }
    const int64_t out = a.c_ptr[col];
    const int32_t col32 = static_cast<int32_t>(col);
    for (int i = lane; i < n; i += kWarp) {
      a.rows[out + i] = sorted[i];
      a.cols[out + i] = col32;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Stage 3: values, one thread per output entry
enum class ValueMode : int { kStore = 0, kResidual = 1, kProjection = 2, kMasked = 3 };

template <class T>
struct ValuesArgs {
  CscView<T> x_csr;
  CscView<T> b;
  const int32_t* rows;
  const int32_t* cols;
  int64_t count;
  int mode;
  bool prune;
  T* out;              // kStore/kResidual: C values; kProjection: t = pr * (X B)
  T* z_out;            // kResidual: Z = pr * R (optional)
  const T* row_scale;  // pr
  double* out_f64;     // kMasked
  int32_t* flag;       // set when a stored value is an exact zero (pruning needed)
};

template <class T>
__global__ void __launch_bounds__(256) ValuesKernel(ValuesArgs<T> a) {
  bool zero_seen = false;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < a.count;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t i = a.rows[p];
    const int32_t j = a.cols[p];
    const int64_t bs = a.b.ptr[j];
    const int blen = static_cast<int>(a.b.ptr[j + 1] - bs);
    const int64_t xs = a.x_csr.ptr[i];
    const int64_t xe = a.x_csr.ptr[i + 1];
    T acc = T(0);  // the storage type's arithmetic (see ColumnProductKernel)
    bool has = false;
    for (int64_t q0 = xs; q0 < xe; q0 += 8) {
      int32_t kk[8];
      T xv[8];
      int64_t at[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int64_t q = q0 + u;
        kk[u] = q < xe ? a.x_csr.idx[q] : INT32_MAX;
        xv[u] = q < xe ? a.x_csr.val[q] : T(0);
        at[u] = bs;
      }
      // eight lower-bound searches in column j of B, in lock step
      int len = blen;
      while (len > 1) {
        const int half = len >> 1;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          if (a.b.idx[at[u] + half] <= kk[u]) at[u] += half;
        }
        len -= half;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (blen > 0 && q0 + u < xe && a.b.idx[at[u]] == kk[u]) {
          const T prod = Mul(xv[u], a.b.val[at[u]]);
          acc = has ? Add(acc, prod) : prod;
          has = true;
        }
      }
    }
    if (a.mode == static_cast<int>(ValueMode::kMasked)) {
      a.out_f64[p] = has ? static_cast<double>(acc) : 0.0;
      continue;
    }
    if (a.mode == static_cast<int>(ValueMode::kProjection)) {
      a.out[p] = Mul(a.row_scale[i], acc);
      continue;
    }
    T v = acc;
    if (a.mode == static_cast<int>(ValueMode::kResidual)) {
      v = has ? -acc : T(0);
      if (i == j) v = has ? Add(v, T(1)) : T(1);
    }
    const T stored = v;
    a.out[p] = stored;
    if (a.z_out != nullptr) a.z_out[p] = Mul(a.row_scale[i], stored);
    if (a.prune && stored == T(0)) zero_seen = true;  // Eigen prune(0.0): +-0 go, NaN stays
  }
  if (__any_sync(0xffffffffu, zero_seen) && (threadIdx.x & 31) == 0) atomicOr(a.flag, 1);
}

// ---------------------------------------------------------------------------
// Stage 4: per-column sequential sums
template <class T>
struct SumsArgs {
  const int64_t* c_ptr;
  const int32_t* rows;
  const T* vals;
  CscView<T> b;  // projection: B = Z
  bool projection;
  double* col_squares;
  double* proj_tt;
  double* proj_bt;
  int64_t cols;
};

template <class T>
__global__ void ColumnSumsKernel(SumsArgs<T> a) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < a.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t s = a.c_ptr[j];
    const int64_t e = a.c_ptr[j + 1];
    double sq = 0.0;
    for (int64_t p = s; p < e; ++p) {
      const double v = static_cast<double>(a.vals[p]);
      sq = Add(sq, Mul(v, v));
    }
    if (!a.projection) {
      a.col_squares[j] = sq;
      continue;
    }
    a.proj_tt[j] = sq;
    double bt = 0.0;
    int64_t p = s;
    int64_t q = a.b.ptr[j];
    const int64_t qe = a.b.ptr[j + 1];
    while (p < e && q < qe) {
      const int32_t r1 = a.rows[p];
      const int32_t r2 = a.b.idx[q];
      if (r1 == r2) {
        bt = Add(bt, Mul(static_cast<double>(a.b.val[q]), static_cast<double>(a.vals[p])));
        ++p;
        ++q;
      } else if (r1 < r2) {
        ++p;
      } else {
        ++q;
      }
    }
    a.proj_bt[j] = bt;
  }
}

// ---------------------------------------------------------------------------
// Column path: stages 1-4 in one warp-per-column kernel for every column
// whose row window fits the bitmap bins.  Per column, in shared memory:
//   * B(:,j) in an open-addressing hash (row -> value);
//   * the output rows in a two-level window bitmap (a summary bit per
//     non-empty 32-row word), read back in ascending order and cleared while
//     it is read, so a column never pays for the empty part of its window;
// then lane r takes output rows r, r+32, ...: walks row i of X (CSR) in
// ascending k, looks each k up in the hash and accumulates the products in
// that order (acc starts at -0.0, so the first addition yields the first
// product exactly: the same bits as "first product, then +=").  Per-column
// sums are sequential in row order (lane 0 over a 32-entry staging buffer).
// C (and Z) are written column by column at padded offsets, exact zeros
// squeezed out when pruning, with counts[j] = the surviving length.
constexpr int kColumnRowsMax = 2048;   // largest output column (upper bound) the column path takes
constexpr int kColumnHashMaxKeys = 1024;

template <class T>
struct ColumnArgs {
  CscView<T> x;      // X by columns: candidate rows
  CscView<T> x_csr;  // X by rows: products in ascending k
  CscView<T> b;
  const int32_t* win_lo;
  const int32_t* win_words;
  bool add_diag;
  int64_t* counts;   // store/residual: surviving length of every column
  int mode;          // ValueMode: kStore, kResidual or kProjection
  bool prune;        // drop exact zeros while writing
  const int64_t* c_ptr;  // padded column offsets (upper bounds)
  int32_t* c_idx;
  T* c_val;
  T* z_val;             // kResidual: Z = pr * R (optional)
  const T* row_scale;   // pr
  double* col_squares;  // optional per-column sum of squares of C
  double* proj_tt;
  double* proj_bt;
  const int32_t* x_cols_ell;  // optional ELL copies of X (see SpgemmExtras)
  const int32_t* x_rows_ell;
  const T* x_rows_ell_val;
  int ell_width;
};


__host__ __device__ inline size_t ColumnSlabBytes(int words, int rows_cap, int hash_slots, size_t value_size) {
  return Round16(static_cast<size_t>(words) * 4) + Round16(static_cast<size_t>(SummaryWords(words)) * 4) +
         Round16(static_cast<size_t>(rows_cap) * 2) + Round16(static_cast<size_t>(hash_slots) * 4) +
         Round16(static_cast<size_t>(hash_slots) * value_size) + 2 * Round16(kWarp * sizeof(double));
}









// kEll: the ELL width of X (compile time, so its loops unroll), 0 without.
template <class T, int kEll>
__global__ void __launch_bounds__(256, 5) ColumnProductKernel(ColumnArgs<T> a, const int32_t* __restrict__ cols_list,
                                                           int64_t list_len, int words_cap, int rows_cap,
                                                           int hash_slots) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int summary_cap = SummaryWords(words_cap);
  unsigned char* base = smem + (threadIdx.x >> 5) * ColumnSlabBytes(words_cap, rows_cap, hash_slots, sizeof(T));
  uint32_t* bm = reinterpret_cast<uint32_t*>(base);
  base += Round16(static_cast<size_t>(words_cap) * 4);
  uint32_t* summary = reinterpret_cast<uint32_t*>(base);
  base += Round16(static_cast<size_t>(summary_cap) * 4);
  uint16_t* rows = reinterpret_cast<uint16_t*>(base);
  base += Round16(static_cast<size_t>(rows_cap) * 2);
  int32_t* hkeys = reinterpret_cast<int32_t*>(base);
  base += Round16(static_cast<size_t>(hash_slots) * 4);
  T* hvals = reinterpret_cast<T*>(base);
  base += Round16(static_cast<size_t>(hash_slots) * sizeof(T));
  double* stage0 = reinterpret_cast<double*>(base);
  double* stage1 = stage0 + kWarp;
  const int hbits = Log2(hash_slots) - 1;  // buckets of two slots
  const bool projection = a.mode == static_cast<int>(ValueMode::kProjection);
  const bool residual = a.mode == static_cast<int>(ValueMode::kResidual);
  const bool sums = projection || a.col_squares != nullptr;
  // both bitmap levels start clear and are left clear by DrainRows
  ClearWords(bm, words_cap, lane);
  ClearWords(summary, summary_cap, lane);
  __syncwarp();
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t at_list = warp; at_list < list_len; at_list += warps) {
    const int64_t col = cols_list[at_list];
    const int words = a.win_words[col];
    const int32_t lo = a.win_lo[col];
    const int64_t bs = a.b.ptr[col];
    const int64_t be = a.b.ptr[col + 1];
    ClearTable(hkeys, hash_slots, lane);
    __syncwarp();
    bool placed = true;
    for (int64_t p = bs + lane; p < be; p += kWarp) placed &= BucketInsert(hkeys, hvals, hbits, a.b.idx[p], a.b.val[p]);
    const bool displaced = !__all_sync(0xffffffffu, placed);
    if (a.add_diag && lane == 0) MarkRow(bm, summary, static_cast<int>(col) - lo);
    if constexpr (kEll > 0) {
      for (int64_t p = bs + lane; p < be; p += kWarp) {
        const int4* src = reinterpret_cast<const int4*>(a.x_cols_ell + static_cast<int64_t>(a.b.idx[p]) * kEll);
#pragma unroll
        for (int u = 0; u < kEll / 4; ++u) {
          const int4 r4 = src[u];
          if (r4.x >= 0) MarkRow(bm, summary, r4.x - lo);
          if (r4.y >= 0) MarkRow(bm, summary, r4.y - lo);
          if (r4.z >= 0) MarkRow(bm, summary, r4.z - lo);
          if (r4.w >= 0) MarkRow(bm, summary, r4.w - lo);
        }
      }
    } else {
      for (int64_t p = bs + lane; p < be; p += kWarp) {
        const int32_t k = a.b.idx[p];
        const int64_t xs = a.x.ptr[k];
        const int64_t xe = a.x.ptr[k + 1];
        for (int64_t q0 = xs; q0 < xe; q0 += 8) {
          int32_t r8[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) r8[u] = q0 + u < xe ? a.x.idx[q0 + u] : -1;
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (r8[u] >= 0) MarkRow(bm, summary, r8[u] - lo);
          }
        }
      }
    }
    __syncwarp();
    const int count = DrainRows(bm, summary, SummaryWords(words), rows, lane);
    const int64_t c0 = projection ? 0 : a.c_ptr[col];
    int kept = 0;
    double sq = 0.0;
    double tt = 0.0;
    double bt = 0.0;
    for (int r0 = 0; r0 < count; r0 += kWarp) {
      const int r = r0 + lane;
      bool have = false;
      int32_t row_out = 0;
      T stored = T(0);
      if (r < count) {
        const int32_t i = lo + static_cast<int32_t>(rows[r]);
        // the storage type's arithmetic: FP64 for double storage, FP32 multiply and accumulate for float storage
        T acc = T(-0.0);
        if constexpr (kEll > 0) {
          const int4* ks = reinterpret_cast<const int4*>(a.x_rows_ell + static_cast<int64_t>(i) * kEll);
          const T* vs = a.x_rows_ell_val + static_cast<int64_t>(i) * kEll;
#pragma unroll
          for (int u = 0; u < kEll / 4; ++u) {
            const int4 k4 = ks[u];
            T v4[4];
            LoadFour(vs + 4 * u, v4);
            const int32_t kk[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              T bv;
              if (kk[e] >= 0 && BucketFind(hkeys, hvals, hbits, displaced, kk[e], bv)) acc = Add(acc, Mul(v4[e], bv));
            }
          }
        } else {
          const int64_t xs = a.x_csr.ptr[i];
          const int64_t xe = a.x_csr.ptr[i + 1];
          for (int64_t q = xs; q < xe; ++q) {
            T bv;
            if (BucketFind(hkeys, hvals, hbits, displaced, a.x_csr.idx[q], bv)) acc = Add(acc, Mul(a.x_csr.val[q], bv));
          }
        }
        if (projection) {
          const double td = static_cast<double>(Mul(a.row_scale[i], acc));
          T zv;
          stage0[lane] = Mul(td, td);
          // rows of Z absent from the product add +0.0, which leaves a sum started at +0.0 unchanged
          stage1[lane] = BucketFind(hkeys, hvals, hbits, displaced, i, zv) ? Mul(static_cast<double>(zv), td) : 0.0;
        } else {
          T v = acc;
          if (residual) {
            v = -acc;
            if (static_cast<int64_t>(i) == col) v = Add(v, T(1));
          }
          stored = v;
          row_out = i;
          have = true;
          const double sd = static_cast<double>(stored);
          stage0[lane] = Mul(sd, sd);
        }
      }
      if (!projection) {
        // Eigen prune(0.0): exact zeros leave C (they add nothing to the column sums)
        const bool keep = have && !(a.prune && stored == T(0));
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const int64_t o = c0 + kept + __popc(mask & LaneMaskBelow());
          a.c_idx[o] = row_out;
          a.c_val[o] = stored;
          if (a.z_val != nullptr) a.z_val[o] = Mul(a.row_scale[row_out], stored);
        }
        kept += __popc(mask);
      }
      if (sums) {
        // sequential in row order; lane 0 sums stage0, lane 1 (projection) stage1
        __syncwarp();
        if (lane < (projection ? 2 : 1)) {
          const double* src = lane == 0 ? stage0 : stage1;
          double s = lane == 0 ? (projection ? tt : sq) : bt;
          const int n = min(kWarp, count - r0);
          if (n == kWarp) {
            const double2* src2 = reinterpret_cast<const double2*>(src);
#pragma unroll
            for (int l = 0; l < kWarp / 2; ++l) {
              const double2 v = src2[l];
              s = Add(s, v.x);
              s = Add(s, v.y);
            }
          } else {
            for (int l = 0; l < n; ++l) s = Add(s, src[l]);
          }
          if (lane == 1) {
            bt = s;
          } else if (projection) {
            tt = s;
          } else {
            sq = s;
          }
        }
        __syncwarp();
      }
    }
    if (projection) {
      if (lane == 0) a.proj_tt[col] = tt;
      if (lane == 1) a.proj_bt[col] = bt;
    } else if (lane == 0) {
      a.counts[col] = kept;
      if (a.col_squares != nullptr) a.col_squares[col] = sq;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Hash need, window and bin of every output column, thread per column (every
// column in flight at once).  Each column is appended to its bin's list (one
// atomic per warp and bin; the fill counters are the bin populations the host
// reads); block-level reduction of the maxima and of the sum of the bounds.
template <class T>
__global__ void __launch_bounds__(256) NeedKernel(CscView<T> x, const int32_t* __restrict__ x_cols_ell, int ell_width,
                                                  CscView<T> b, bool add_diag, int64_t* __restrict__ need,
                                                  int64_t* __restrict__ ub, int32_t* __restrict__ win_lo,
                                                  int32_t* __restrict__ win_words, int32_t* __restrict__ bin_cols,
                                                  unsigned long long* __restrict__ maxima) {
  __shared__ unsigned long long block_max[3];  // max ub, max nnz(B col), sum of ub
  if (threadIdx.x < 3) block_max[threadIdx.x] = 0ull;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  unsigned long long local_ub = 0;
  unsigned long long local_nb = 0;
  unsigned long long local_sum = 0;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x; base < b.cols;
       base += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t j = base + threadIdx.x;
    int bin = -1;  // every lane takes part in the ballots below, columns past the end included
    if (j < b.cols) {
      const int64_t bs = b.ptr[j];
      const int64_t be = b.ptr[j + 1];
      int64_t u = add_diag ? 1 : 0;
      int32_t lo = add_diag ? static_cast<int32_t>(j) : INT32_MAX;
      int32_t hi = add_diag ? static_cast<int32_t>(j) : -1;
      for (int64_t p = bs; p < be; ++p) {
        const int32_t k = b.idx[p];
        if (ell_width > 0) {
          // the ELL copy of X(:,k): its rows in ascending order, then -1 padding
          const int4* e = reinterpret_cast<const int4*>(x_cols_ell + static_cast<int64_t>(k) * ell_width);
          for (int q = 0; q < ell_width / 4; ++q) {
            const int4 r4 = e[q];
            const int32_t r[4] = {r4.x, r4.y, r4.z, r4.w};
#pragma unroll
            for (int t = 0; t < 4; ++t) {
              if (r[t] >= 0) {
                ++u;
                lo = min(lo, r[t]);
                hi = max(hi, r[t]);
              }
            }
          }
        } else {
          const int64_t xs = x.ptr[k];
          const int64_t xe = x.ptr[k + 1];
          if (xe > xs) {
            u += xe - xs;
            lo = min(lo, x.idx[xs]);
            hi = max(hi, x.idx[xe - 1]);
          }
        }
      }
      int words = 0;
      if (hi >= lo) {
        const int64_t w = (static_cast<int64_t>(hi) - lo) / 32 + 1;
        words = w > INT32_MAX ? INT32_MAX : static_cast<int>(w);
      }
      need[j] = 2 * u;
      ub[j] = u;
      win_lo[j] = hi >= lo ? lo : 0;
      win_words[j] = words;
      // bins: <= 128, 512, 1040, 2048 words (kWordBins), else the hash path
      bin = words <= 128 ? 0 : (words <= 512 ? 1 : (words <= 1040 ? 2 : (words <= kBitmapMaxWords ? 3 : 4)));
      local_sum += static_cast<unsigned long long>(u);
      local_ub = max(local_ub, static_cast<unsigned long long>(u));
      local_nb = max(local_nb, static_cast<unsigned long long>(be - bs));
    }
#pragma unroll
    for (int i = 0; i <= kWordBinCount; ++i) {
      const unsigned mask = __ballot_sync(0xffffffffu, bin == i);
      if (mask == 0u) continue;
      const int leader = __ffs(mask) - 1;
      unsigned long long first = 0ull;
      unsigned long long* fill = i < kWordBinCount ? &maxima[kPopulation + i] : &maxima[kHashColumns];
      if (lane == leader) first = atomicAdd(fill, static_cast<unsigned long long>(__popc(mask)));
      first = __shfl_sync(0xffffffffu, first, leader);
      if (bin == i) {
        bin_cols[static_cast<int64_t>(i) * b.cols + static_cast<int64_t>(first) + __popc(mask & LaneMaskBelow())] =
            static_cast<int32_t>(j);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    local_ub = max(local_ub, __shfl_xor_sync(0xffffffffu, local_ub, o));
    local_nb = max(local_nb, __shfl_xor_sync(0xffffffffu, local_nb, o));
    local_sum += __shfl_xor_sync(0xffffffffu, local_sum, o);
  }
  if (lane == 0) {
    atomicMax(&block_max[0], local_ub);
    atomicMax(&block_max[1], local_nb);
    if (local_sum != 0ull) atomicAdd(&block_max[2], local_sum);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (block_max[0] != 0ull) atomicMax(&maxima[kMaxUb], block_max[0]);
    if (block_max[1] != 0ull) atomicMax(&maxima[kMaxNb], block_max[1]);
    if (block_max[2] != 0ull) atomicAdd(&maxima[kSumUb], block_max[2]);
  }
}

template <class T>
__global__ void ColumnIdsKernel(CscView<T> m, int32_t* __restrict__ cols) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < m.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    for (int64_t p = m.ptr[j]; p < m.ptr[j + 1]; ++p) cols[p] = static_cast<int32_t>(j);
  }
}

struct HashBin {
  int slots;
  int warps;
  int64_t lo;
  int64_t hi;
};

constexpr HashBin kHashBins[] = {
    {256, 8, -1, 256},
    {1024, 8, 256, 1024},
    {4096, 4, 1024, 4096},
};
constexpr int64_t kLargestHashBin = 4096;

int NextPow2(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return static_cast<int>(p);
}

int WarpsFor(size_t bytes_per_warp) {
  const size_t budget = 96 * 1024;
  int warps = static_cast<int>(budget / (bytes_per_warp > 0 ? bytes_per_warp : 1));
  return warps < 1 ? 1 : (warps > 16 ? 16 : warps);
}

// Launches the row-set stage (count or list mode) over every populated bin.
template <class T>
void LaunchRowSets(Ctx& ctx, RowSetArgs<T> args, const unsigned long long* host_max) {
  int lo_words = -1;
  for (int bin = 0; bin < kWordBinCount; ++bin) {
    const int words_cap = kWordBins[bin];
    const int64_t population = static_cast<int64_t>(host_max[kPopulation + bin]);
    if (population > 0) {
      const size_t per_warp = BitmapBytes(words_cap);
      const int warps = WarpsFor(per_warp);
      const size_t smem = per_warp * warps;
      SPAI_CUDA(cudaFuncSetAttribute(BitmapRowSetKernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
      BitmapRowSetKernel<T><<<GridFor(population * kWarp, warps * kWarp), warps * kWarp, smem, ctx.stream>>>(
          args, words_cap, lo_words, words_cap);
      SPAI_LAUNCH_CHECK();
    }
    lo_words = words_cap;
  }
  if (host_max[kHashColumns] == 0) return;
  const int64_t max_need = 2 * static_cast<int64_t>(host_max[kMaxUb]);
  const int64_t hash_columns = static_cast<int64_t>(host_max[kHashColumns]);
  for (const HashBin& bin : kHashBins) {
    if (max_need <= bin.lo) break;
    const size_t smem = HashRowSetBytes(bin.slots) * bin.warps;
    SPAI_CUDA(cudaFuncSetAttribute(HashRowSetKernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    const int threads = bin.warps * kWarp;
    args.global_space = nullptr;
    HashRowSetKernel<T><<<GridFor(hash_columns * kWarp, threads), threads, smem, ctx.stream>>>(args, bin.slots, bin.lo,
                                                                                            bin.hi);
    SPAI_LAUNCH_CHECK();
  }
  if (max_need > kLargestHashBin) {
    const int slots = NextPow2(max_need);
    const int blocks = ctx.sm_count * 2;
    ctx.sg_fallback.Reserve(HashRowSetBytes(slots) * blocks, ctx.stream);
    args.global_space = ctx.sg_fallback.data();
    HashRowSetKernel<T><<<blocks, kWarp, 0, ctx.stream>>>(args, slots, kLargestHashBin, INT64_MAX);
    SPAI_LAUNCH_CHECK();
  }
}

// Warps per block of a warp-per-column kernel with `per_warp` bytes of shared
// memory per warp: the count that keeps the most warps resident per SM (the
// slab makes shared memory the usual limit, in steps of a block).  Cached per
// kernel and slab size.
int WarpsPerBlock(const void* kernel, size_t per_warp) {
  static std::mutex mutex;
  static std::map<std::pair<const void*, size_t>, int> chosen;
  std::lock_guard<std::mutex> lock(mutex);
  const auto key = std::make_pair(kernel, per_warp);
  const auto it = chosen.find(key);
  if (it != chosen.end()) return it->second;
  int warps = 1;
  int best_resident = -1;
  for (int w = 8; w >= 1; --w) {
    const size_t bytes = per_warp * static_cast<size_t>(w);
    if (bytes > static_cast<size_t>(200 * 1024)) continue;
    SPAI_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    int blocks = 0;
    SPAI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, w * kWarp, bytes));
    if (blocks * w > best_resident) {
      best_resident = blocks * w;
      warps = w;
    }
  }
  chosen[key] = warps;
  return warps;
}

// Block sizes of the column kernel, chosen by timing.  The first launch of a
// (kernel, shared-memory slab) pair over at least kTuneMinColumns columns runs
// the bin once with every block size whose slabs fit (1, 2, 4 or 8 warps),
// timed with CUDA events on the launching stream; the fastest is kept for the
// process.  The kernel writes the same outputs whatever its block size, so
// the trial launches change no result.  Smaller launches use the block size
// of highest occupancy until a tuned one exists.
constexpr int64_t kTuneMinColumns = 8192;

struct TunedWarps {
  std::mutex mutex;
  std::map<std::pair<const void*, size_t>, int> chosen;
};

TunedWarps& Tuned() {
  static TunedWarps* table = new TunedWarps();  // kept for the process: launches may run during exit
  return *table;
}

int LookUpTuned(const void* kernel, size_t per_warp) {
  TunedWarps& t = Tuned();
  std::lock_guard<std::mutex> lock(t.mutex);
  const auto it = t.chosen.find(std::make_pair(kernel, per_warp));
  return it == t.chosen.end() ? 0 : it->second;
}

// The column path: one launch per populated bitmap bin, over that bin's
// column list (written by NeedKernel), with the bin's shared-memory layout.
template <class T>
void LaunchColumnProducts(Ctx& ctx, const ColumnArgs<T>& args, const unsigned long long* host_max, int rows_cap,
                          int hash_slots) {
  for (int bin = 0; bin < kWordBinCount; ++bin) {
    const int64_t population = static_cast<int64_t>(host_max[kPopulation + bin]);
    if (population == 0) continue;
    const int words_cap = kWordBins[bin];
    const size_t per_warp = ColumnSlabBytes(words_cap, rows_cap, hash_slots, sizeof(T));
    void (*kernel)(ColumnArgs<T>, const int32_t*, int64_t, int, int, int) = ColumnProductKernel<T, 0>;
    switch (args.ell_width) {
      case 4: kernel = ColumnProductKernel<T, 4>; break;
      case 8: kernel = ColumnProductKernel<T, 8>; break;
      case 12: kernel = ColumnProductKernel<T, 12>; break;
      case 16: kernel = ColumnProductKernel<T, 16>; break;
      default: break;
    }
    const int32_t* list = ctx.sg_bin_cols.data() + static_cast<int64_t>(bin) * args.b.cols;
    const void* key = reinterpret_cast<const void*>(kernel);
    auto launch = [&](int warps) {
      const size_t smem = per_warp * static_cast<size_t>(warps);
      SPAI_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
      kernel<<<GridFor(population * kWarp, warps * kWarp), warps * kWarp, smem, ctx.stream>>>(
          args, list, population, words_cap, rows_cap, hash_slots);
      SPAI_LAUNCH_CHECK();
    };
    int warps = LookUpTuned(key, per_warp);
    if (warps == 0 && population >= kTuneMinColumns) {
      cudaEvent_t start = nullptr;
      cudaEvent_t stop = nullptr;
      SPAI_CUDA(cudaEventCreate(&start));
      SPAI_CUDA(cudaEventCreate(&stop));
      float best_ms = 0.0f;
      for (int w = 1; w <= 8; w <<= 1) {
        const size_t bytes = per_warp * static_cast<size_t>(w);
        if (bytes > static_cast<size_t>(200 * 1024)) break;
        SPAI_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
        int blocks = 0;
        SPAI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, w * kWarp, bytes));
        if (blocks < 1) break;
        SPAI_CUDA(cudaEventRecord(start, ctx.stream));
        launch(w);
        SPAI_CUDA(cudaEventRecord(stop, ctx.stream));
        SPAI_CUDA(cudaEventSynchronize(stop));
        float ms = 0.0f;
        SPAI_CUDA(cudaEventElapsedTime(&ms, start, stop));
        if (warps == 0 || ms < best_ms) {
          best_ms = ms;
          warps = w;
        }
      }
      cudaEventDestroy(start);
      cudaEventDestroy(stop);
      if (warps != 0) {
        TunedWarps& t = Tuned();
        std::lock_guard<std::mutex> lock(t.mutex);
        t.chosen[std::make_pair(key, per_warp)] = warps;
        continue;  // the trial launches already wrote this bin's outputs
      }
    }
    if (warps == 0) warps = WarpsPerBlock(key, per_warp);
    launch(warps);
  }
}

template <class T>
double MatrixBytes(int64_t nnz, int64_t major) {
  return static_cast<double>(nnz) * static_cast<double>(sizeof(T) + sizeof(int32_t)) +
         static_cast<double>(major + 1) * static_cast<double>(sizeof(int64_t));
}

}  // namespace

template <class T>
bool Spgemm(Ctx& ctx, const DevCsc<T>& x_csc, const DevCsc<T>& x_csr, const DevCsc<T>& b, DevCsc<T>& c,
            Epilogue epilogue, SpgemmExtras extras, DevCsc<T>* c_z) {
  const int64_t cols = b.cols;
  const bool residual = epilogue == Epilogue::kResidual;
  const bool projection = epilogue == Epilogue::kProjection;
  ctx.sg_need.Reserve(static_cast<size_t>(cols), ctx.stream);
  ctx.sg_counts.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
  ctx.sg_win_lo.Reserve(static_cast<size_t>(cols), ctx.stream);
  ctx.sg_win_words.Reserve(static_cast<size_t>(cols), ctx.stream);
  ctx.sg_maxima.Reserve(kMaximaSlots, ctx.stream);
  ctx.sg_bin_cols.Reserve(static_cast<size_t>(kWordBinCount + 1) * static_cast<size_t>(cols), ctx.stream);
  SPAI_CUDA(cudaMemsetAsync(ctx.sg_maxima.data(), 0, kMaximaSlots * sizeof(unsigned long long), ctx.stream));
  NeedKernel<T><<<GridFor(cols, 256), 256, 0, ctx.stream>>>(View(x_csc), extras.x_cols_ell, extras.ell_width, View(b),
                                                            residual,
                                                                   ctx.sg_need.data(), ctx.sg_counts.data(),
                                                                   ctx.sg_win_lo.data(), ctx.sg_win_words.data(),
                                                                   ctx.sg_bin_cols.data(), ctx.sg_maxima.data());
  SPAI_LAUNCH_CHECK();
  unsigned long long host_max[kMaximaSlots];
  SPAI_CUDA(cudaMemcpyAsync(host_max, ctx.sg_maxima.data(), sizeof(host_max), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();

  const int64_t max_u = static_cast<int64_t>(host_max[kMaxUb]);
  const int64_t max_nb = static_cast<int64_t>(host_max[kMaxNb]);
  const bool column_path =
      host_max[kHashColumns] == 0 && max_u <= kColumnRowsMax && max_nb <= kColumnHashMaxKeys;
  const ValueMode mode = residual ? ValueMode::kResidual : (projection ? ValueMode::kProjection : ValueMode::kStore);
  const bool prune = epilogue == Epilogue::kPruneZeros || residual;
  const bool want_z = residual && extras.row_scale != nullptr && c_z != nullptr;
  // algorithmic bytes: |X| + |B| + |C| (the projection writes per-column sums instead of C)
  const double operand_bytes = MatrixBytes<T>(x_csr.nnz, x_csr.cols) + MatrixBytes<T>(b.nnz, b.cols);

  ColumnArgs<T> ca{};
  ca.x = View(x_csc);
  ca.x_csr = View(x_csr);
  ca.b = View(b);
  ca.win_lo = ctx.sg_win_lo.data();
  ca.win_words = ctx.sg_win_words.data();
  ca.add_diag = residual;
  ca.mode = static_cast<int>(mode);
  ca.prune = prune;
  ca.row_scale = static_cast<const T*>(extras.row_scale);
  ca.col_squares = extras.col_squares;
  ca.proj_tt = extras.proj_tt;
  ca.proj_bt = extras.proj_bt;
  ca.x_cols_ell = extras.x_cols_ell;
  ca.x_rows_ell = extras.x_rows_ell;
  ca.x_rows_ell_val = static_cast<const T*>(extras.x_rows_ell_val);
  ca.ell_width = extras.ell_width;
  const int rows_cap = NextPow2(max_u > kWarp ? max_u : kWarp);
  // load factor <= 1/4 while the table stays small, <= 1/2 beyond
  const int hash_slots = NextPow2(4 * max_nb <= 1024 ? (4 * max_nb > kWarp ? 4 * max_nb : kWarp) : 2 * max_nb);

  if (projection && column_path) {
    // no output matrix: no count pass, no scan, no host round trip
    prof::Scope scope(ctx.stream, "spgemm_numeric",
                      operand_bytes + static_cast<double>(cols) * (sizeof(T) + 2 * sizeof(double)));
    LaunchColumnProducts(ctx, ca, host_max, rows_cap, hash_slots);
    return false;
  }
  if (column_path) {
    // one pass into padded columns (offsets: scan of the upper bounds NeedKernel left in sg_counts),
    // then one scan of the surviving lengths and a compaction
    const int64_t padded = static_cast<int64_t>(host_max[kSumUb]);
    const size_t slots = static_cast<size_t>(padded > 0 ? padded : 1);
    ctx.sg_ub_ptr.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
    ctx.sg_pad_idx.Reserve(slots, ctx.stream);
    ctx.sg_pad_val.Reserve(slots * sizeof(T), ctx.stream);
    if (want_z) ctx.sg_pad_z.Reserve(slots * sizeof(T), ctx.stream);
    ScanCountsAsync(ctx, ctx.sg_counts.data(), cols, ctx.sg_ub_ptr.data());
    T* pad_val = reinterpret_cast<T*>(ctx.sg_pad_val.data());
    T* pad_z = want_z ? reinterpret_cast<T*>(ctx.sg_pad_z.data()) : nullptr;
    ca.c_ptr = ctx.sg_ub_ptr.data();
    ca.c_idx = ctx.sg_pad_idx.data();
    ca.c_val = pad_val;
    ca.z_val = pad_z;
    ca.counts = ctx.sg_counts.data();
    DevCsc<T> result;
    result.Shape(x_csc.rows, cols, ctx.stream);
    int64_t nnz = 0;
    {
      prof::Scope scope(ctx.stream, "spgemm_numeric", 0.0);
      LaunchColumnProducts(ctx, ca, host_max, rows_cap, hash_slots);
    }
    nnz = ScanCounts(ctx, ctx.sg_counts.data(), cols, result.ptr.data());
    result.ReserveNnz(nnz, ctx.stream);
    {
      // the numeric pass: |X| + |B| read, C (and Z, the column sums) written once
      double bytes = operand_bytes + MatrixBytes<T>(nnz, cols);
      if (want_z) bytes += static_cast<double>(nnz) * sizeof(T);
      if (extras.col_squares != nullptr) bytes += static_cast<double>(cols) * sizeof(double);
      prof::AddBytes("spgemm_numeric", bytes);
    }
    {
      // the compaction reads and writes C (and Z) once more
      double bytes = 2.0 * MatrixBytes<T>(nnz, cols);
      if (want_z) bytes += 2.0 * static_cast<double>(nnz) * (sizeof(T) + sizeof(int32_t));
      prof::Scope scope(ctx.stream, "spgemm_compact", bytes);
      if (want_z) {
        DevCsc<T> z;
        z.Shape(result.rows, cols, ctx.stream);
        z.ReserveNnz(nnz, ctx.stream);
        SPAI_CUDA(cudaMemcpyAsync(z.ptr.data(), result.ptr.data(), sizeof(int64_t) * (cols + 1),
                                  cudaMemcpyDeviceToDevice, ctx.stream));
        CompactPaddedPair(ctx, ctx.sg_ub_ptr.data(), cols, result.ptr.data(), ctx.sg_pad_idx.data(), pad_val,
                          result.idx.data(), result.val.data(), static_cast<const T*>(pad_z), z.idx.data(),
                          z.val.data());
        c_z->Swap(z);
      } else {
        CompactPadded(ctx, ctx.sg_ub_ptr.data(), static_cast<const int64_t*>(nullptr), cols, result.ptr.data(),
                      ctx.sg_pad_idx.data(), pad_val, result.idx.data(), result.val.data());
      }
    }
    c.Swap(result);
    return want_z;
  }

  RowSetArgs<T> rs{};
  rs.x = View(x_csc);
  rs.b = View(b);
  rs.need = ctx.sg_need.data();
  rs.win_lo = ctx.sg_win_lo.data();
  rs.win_words = ctx.sg_win_words.data();
  rs.add_diag = residual;
  rs.counts = ctx.sg_counts.data();
  {
    prof::Scope scope(ctx.stream, "spgemm_symbolic", 0.0);
    rs.list = false;
    LaunchRowSets(ctx, rs, host_max);
  }

  // output layout: C, or the transient row list of the projection
  DevCsc<T> result;
  int64_t* c_ptr;
  if (projection) {
    ctx.sg_proj_ptr.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
    c_ptr = ctx.sg_proj_ptr.data();
  } else {
    result.Shape(x_csc.rows, cols, ctx.stream);
    c_ptr = result.ptr.data();
  }
  const int64_t nnz = ScanCounts(ctx, ctx.sg_counts.data(), cols, c_ptr);
  int32_t* rows;
  T* vals;
  if (projection) {
    ctx.sg_proj_rows.Reserve(static_cast<size_t>(nnz > 0 ? nnz : 1), ctx.stream);
    ctx.sg_proj_vals.Reserve(static_cast<size_t>(nnz > 0 ? nnz : 1) * sizeof(T), ctx.stream);
    rows = ctx.sg_proj_rows.data();
    vals = reinterpret_cast<T*>(ctx.sg_proj_vals.data());
  } else {
    result.ReserveNnz(nnz, ctx.stream);
    rows = result.idx.data();
    vals = result.val.data();
  }
  DevBuf<T> zbuf;
  if (want_z) zbuf.Reserve(static_cast<size_t>(nnz > 0 ? nnz : 1), ctx.stream);
  SPAI_CUDA(cudaMemsetAsync(ctx.flags.data(), 0, sizeof(int32_t), ctx.stream));
  {
    double bytes = operand_bytes;
    if (projection) {
      bytes += static_cast<double>(cols) * (sizeof(T) + 2 * sizeof(double));
    } else {
      bytes += MatrixBytes<T>(nnz, cols);
      if (want_z) bytes += static_cast<double>(nnz) * sizeof(T);
      if (extras.col_squares != nullptr) bytes += static_cast<double>(cols) * sizeof(double);
    }
    prof::Scope scope(ctx.stream, "spgemm_numeric", bytes);
    {
      ctx.sg_cols.Reserve(static_cast<size_t>(nnz > 0 ? nnz : 1), ctx.stream);
      rs.list = true;
      rs.c_ptr = c_ptr;
      rs.rows = rows;
      rs.cols = ctx.sg_cols.data();
      LaunchRowSets(ctx, rs, host_max);
      ValuesArgs<T> va{};
      va.x_csr = View(x_csr);
      va.b = View(b);
      va.rows = rows;
      va.cols = ctx.sg_cols.data();
      va.count = nnz;
      va.mode = static_cast<int>(mode);
      va.prune = prune;
      va.out = vals;
      va.z_out = want_z ? zbuf.data() : nullptr;
      va.row_scale = static_cast<const T*>(extras.row_scale);
      va.flag = ctx.flags.data();
      if (nnz > 0) {
        ValuesKernel<T><<<GridFor(nnz, 256), 256, 0, ctx.stream>>>(va);
        SPAI_LAUNCH_CHECK();
      }
      if (projection || extras.col_squares != nullptr) {
        SumsArgs<T> sa{c_ptr, rows, vals, View(b), projection, extras.col_squares, extras.proj_tt, extras.proj_bt,
                       cols};
        ColumnSumsKernel<T><<<GridFor(cols, 128), 128, 0, ctx.stream>>>(sa);
        SPAI_LAUNCH_CHECK();
      }
    }
  }
  if (projection) return false;
  bool z_written = want_z;
  if (prune) {
    SPAI_CUDA(cudaMemcpyAsync(ctx.host_flags, ctx.flags.data(), sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.Sync();
    if (ctx.host_flags[0] != 0) {
      // an exact zero: prune it (Eigen prune(0.0)); the fused Z is dropped and recomputed by the caller
      DropZeros(ctx, result);
      z_written = false;
    }
  }
  if (z_written) {
    DevCsc<T> z;
    z.Shape(result.rows, cols, ctx.stream);
    z.ReserveNnz(result.nnz, ctx.stream);
    SPAI_CUDA(cudaMemcpyAsync(z.ptr.data(), result.ptr.data(), sizeof(int64_t) * (cols + 1), cudaMemcpyDeviceToDevice,
                              ctx.stream));
    if (result.nnz > 0) {
      SPAI_CUDA(cudaMemcpyAsync(z.idx.data(), result.idx.data(), sizeof(int32_t) * result.nnz,
                                cudaMemcpyDeviceToDevice, ctx.stream));
    }
    z.val.Swap(zbuf);
    c_z->Swap(z);
  }
  c.Swap(result);
  return z_written;
}

template <class T>
void SpgemmMasked(Ctx& ctx, const DevCsc<T>& x_csr, const DevCsc<T>& b, const DevCsc<T>& mask, double* out) {
  if (mask.nnz == 0) return;
  ctx.sg_cols.Reserve(static_cast<size_t>(mask.nnz), ctx.stream);
  ColumnIdsKernel<T><<<GridFor(mask.cols, 128), 128, 0, ctx.stream>>>(View(mask), ctx.sg_cols.data());
  SPAI_LAUNCH_CHECK();
  ValuesArgs<T> va{};
  va.x_csr = View(x_csr);
  va.b = View(b);
  va.rows = mask.idx.data();
  va.cols = ctx.sg_cols.data();
  va.count = mask.nnz;
  va.mode = static_cast<int>(ValueMode::kMasked);
  va.out_f64 = out;
  va.flag = ctx.flags.data();
  ValuesKernel<T><<<GridFor(mask.nnz, 256), 256, 0, ctx.stream>>>(va);
  SPAI_LAUNCH_CHECK();
}

template bool Spgemm<double>(Ctx&, const DevCsc<double>&, const DevCsc<double>&, const DevCsc<double>&,
                             DevCsc<double>&, Epilogue, SpgemmExtras, DevCsc<double>*);
template bool Spgemm<float>(Ctx&, const DevCsc<float>&, const DevCsc<float>&, const DevCsc<float>&, DevCsc<float>&,
                            Epilogue, SpgemmExtras, DevCsc<float>*);
template void SpgemmMasked<double>(Ctx&, const DevCsc<double>&, const DevCsc<double>&, const DevCsc<double>&,
                                   double*);
template void SpgemmMasked<float>(Ctx&, const DevCsc<float>&, const DevCsc<float>&, const DevCsc<float>&, double*);

}  // namespace spai
