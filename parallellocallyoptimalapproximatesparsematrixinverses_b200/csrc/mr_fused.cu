// The fused, graph-captured Global MR iteration (mr_fused.cuh).
//
// Slot layouts (all in HBM, sized once per solver):
//   M    topk slots per column, rows ascending, count per column
//   M^T  two sets (the drop kernel reads one and writes the other), cap_mt
//        slots per row in arrival order, count per row
//   Z    cap_z slots per column, rows ascending (Z = Pr R keeps R's pattern)
// Z is never transposed: the drop kernel needs row j of Z only for column j,
// and forms it from the rows of M it has (M^T) and row j of A, with the same
// products in the same order as the residual kernel's column of R.  The
// residual kernel clears the M^T set the drop kernel has just read, so the
// next drop kernel fills it again from zero.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <vector>

#include "colkit.cuh"
#include "device.cuh"
#include "mr_fused.cuh"
#include "ops.cuh"
#include "profile.cuh"
#include "select.cuh"
#include "tree.cuh"

namespace spai {

void CountLaunches(int64_t count);

namespace {

constexpr int kDropWarps = 4;       // warps per block of the drop kernel
constexpr int kDropWindowWords = 512;  // bitmap words of the drop kernel: windows of 16,384 rows
constexpr int kDropWindowRows = kDropWindowWords * 32;
constexpr int kResidualWarps = 4;   // warps per block of the residual kernel
constexpr int kWindowWords = 1024;  // bitmap words of the residual kernel: windows of 32,768 rows
constexpr int kWindowRows = kWindowWords * 32;
constexpr int kRowsCap = 1024;      // longest row list of one product column
constexpr int kMaxTopK = 32;
constexpr int kDropRowsCap = 512;  // candidate rows of one drop column; also bounds Z's slots per column

// Overflow bits (FusedState::overflow).
constexpr int kOverflowMt = 1;      // a row of M^T exceeded cap_mt
constexpr int kOverflowRow = 2;     // row j of R had more entries than its hash takes
constexpr int kOverflowSide = 4;    // a drop column's merged rows exceeded kDropCap

// Stop codes (FusedState::stop).
constexpr int kRunning = 0;
constexpr int kConverged = 1;
constexpr int kBreakdown = 2;
constexpr int kIterationLimit = 3;
constexpr int kOverflowStop = 4;

struct FusedRow {
  int64_t iteration;
  double residual_norm;
  double density_m;
  double density_direction;
};

// Device-resident loop state.
struct FusedState {
  double alpha;                 // step length of the next iteration
  int64_t iteration;            // last history row appended
  int64_t parity;               // M^T set the next drop kernel reads
  unsigned long long nnz_m;     // entries of M written by this iteration's drop kernel
  unsigned long long nnz_z;     // entries of Z written by this iteration's residual kernel
  unsigned long long nnz_dir;   // entries of the Z this iteration's step used (its history row's direction)
  unsigned long long last_nnz_m;  // the last iteration's counts (read by the host when profiling)
  unsigned long long last_nnz_z;
  int32_t overflow;
  int32_t stop;
  unsigned int arrive;          // blocks of the decide kernel that are done
  int32_t pad;
  int64_t bodies;               // loop-body executions
};

template <class T>
struct FusedArgs {
  int64_t n;
  int topk;
  int cap_z;
  int cap_mt;
  int ell;  // ELL slots of A (multiple of 4)
  int m_hash_slots;   // residual kernel: M(:, j)
  int z_hash_slots;   // residual kernel: Z(:, j)
  int d_mt_slots;     // drop kernel: M(j, :)
  int d_r_slots;      // drop kernel: R(j, :)
  int64_t max_iterations;
  double tolerance;
  const int32_t* a_cols_ell;
  const int32_t* a_rows_ell;
  const T* a_rows_ell_val;
  const T* pr;
  int32_t* m_rows;
  T* m_vals;
  int32_t* m_cnt;
  int32_t* mt_cols[2];
  T* mt_vals[2];
  int32_t* mt_cnt[2];
  int32_t* z_rows;
  T* z_vals;
  int32_t* z_cnt;
  double* sq;          // per-column sum of squares of R
  double* tt;          // per-column ||Pr A Z(:, j)||^2
  double* bt;          // per-column <Z(:, j), Pr A Z(:, j)>
  double* chunk;       // 3 * chunks
  FusedRow* history;   // max_iterations + 1 rows
  FusedState* state;
};

// ---------------------------------------------------------------------------
// Drop kernel: per column j, S = 0.5 (U(:, j) + U(j, :)^T) with U = M + alpha Z.
//
// M(:, j) and Z(:, j) are read from the column's sorted slots (binary
// searches); two small hashes in shared memory hold M(j, :) (row j of M, from
// M^T) and R(j, :).  Row j of R is formed
// here: for the entries k of row j of A in ascending order, every entry
// M(k, i) of row k of M adds A(j, k) M(k, i) to R(j, i) -- for each i the
// terms arrive in ascending k, exactly the sum the residual kernel forms for
// R(j, i) in column i.  The candidate rows i of S(:, j) (the rows of M(:, j)
// and Z(:, j), the keys of the two hashes, and j) are marked in a window
// bitmap and read back in ascending order; each one's U(i, j), U(j, i) and
// S(i, j) come from those lookups, with
// the union's and the symmetrisation's arithmetic (UnionPadded,
// SymmetrizeDropKernel).  Exact zeros of U are not pruned here: an entry that
// is zero on both sides gives S(i, j) = 0, which the drop rule removes, and a
// zero on one side gives the same half sum as an absent one, so the kept
// entries and their order are the unfused kernels'.

// Returns the slot of key (inserted when absent: *fresh), or -1 when the table is full.
__device__ __forceinline__ int FindOrInsert(int32_t* keys, int bits, int32_t key, bool* fresh) {
  const uint32_t mask = (1u << bits) - 1u;
  uint32_t h = (static_cast<uint32_t>(key) * 2654435761u) >> (32 - bits);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const int32_t old = atomicCAS(&keys[h], kEmpty, key);
    if (old == kEmpty) {
      *fresh = true;
      return static_cast<int>(h);
    }
    if (old == key) {
      *fresh = false;
      return static_cast<int>(h);
    }
    h = (h + 1u) & mask;
  }
  *fresh = false;
  return -1;
}

__device__ __forceinline__ int FindSlot(const int32_t* keys, int bits, int32_t key) {
  const uint32_t mask = (1u << bits) - 1u;
  uint32_t h = (static_cast<uint32_t>(key) * 2654435761u) >> (32 - bits);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const int32_t k = keys[h];
    if (k == key) return static_cast<int>(h);
    if (k == kEmpty) return -1;
    h = (h + 1u) & mask;
  }
  return -1;
}

// Entries of one row of M^T a lane holds while row j of R is formed (cap_mt <= 4 * kMaxTopK).
constexpr int kMtPerLane = 4;
static_assert(4 * kMaxTopK <= kMtPerLane * kWarp, "a row of M^T must fit the lanes' registers");

template <class T>
__host__ __device__ size_t DropWarpBytes(int own, int mt, int r) {
  constexpr int kSummary = (kDropWindowWords + kWarp * kWarp - 1) / (kWarp * kWarp) * kWarp;
  return Round16(static_cast<size_t>(kDropWindowWords) * 4) + Round16(static_cast<size_t>(kSummary) * 4) +
         Round16(static_cast<size_t>(kDropRowsCap) * 2) +
         Round16(static_cast<size_t>(mt + r) * 4) + Round16(static_cast<size_t>(mt + r) * sizeof(T)) +
         Round16(static_cast<size_t>(own) * 4) + Round16(static_cast<size_t>(own) * sizeof(T)) +
         Round16(kDropCap * sizeof(double)) + Round16(kDropCap * sizeof(int32_t)) + Round16(kDropCap) +
         Round16(4 * kWarp * sizeof(int32_t));
}

template <class T>
__global__ void __launch_bounds__(kDropWarps * kWarp) FusedDropKernel(FusedArgs<T> a) {
  extern __shared__ __align__(16) unsigned char fused_drop_smem[];
  constexpr int kSummary = (kDropWindowWords + kWarp * kWarp - 1) / (kWarp * kWarp) * kWarp;
  const int lane = threadIdx.x & 31;
  const int table = a.d_mt_slots + a.d_r_slots;
  const int own = a.topk + a.cap_z;  // M(:, j) and Z(:, j), staged
  unsigned char* base = fused_drop_smem + (threadIdx.x >> 5) * DropWarpBytes<T>(own, a.d_mt_slots, a.d_r_slots);
  uint32_t* bm = reinterpret_cast<uint32_t*>(base);
  base += Round16(static_cast<size_t>(kDropWindowWords) * 4);
  uint32_t* summary = reinterpret_cast<uint32_t*>(base);
  base += Round16(static_cast<size_t>(kSummary) * 4);
  uint16_t* rows = reinterpret_cast<uint16_t*>(base);
  base += Round16(static_cast<size_t>(kDropRowsCap) * 2);
  int32_t* keys = reinterpret_cast<int32_t*>(base);  // the two tables, one after another
  base += Round16(static_cast<size_t>(table) * 4);
  T* vals = reinterpret_cast<T*>(base);
  base += Round16(static_cast<size_t>(table) * sizeof(T));
  int32_t* mr = reinterpret_cast<int32_t*>(base);  // M(:, j) then Z(:, j): rows
  int32_t* zr = mr + a.topk;
  base += Round16(static_cast<size_t>(own) * 4);
  T* mv = reinterpret_cast<T*>(base);  // and values
  T* zv = mv + a.topk;
  base += Round16(static_cast<size_t>(own) * sizeof(T));
  DropSlab s;
  s.vals = reinterpret_cast<double*>(base);
  base += Round16(kDropCap * sizeof(double));
  s.keys = reinterpret_cast<int32_t*>(base);
  base += Round16(kDropCap * sizeof(int32_t));
  s.keep = base;
  base += Round16(kDropCap);
  s.xk = reinterpret_cast<int32_t*>(base);  // staging of the top-k selection
  s.yk = s.xk;
  s.mx_prefix = nullptr;
  int32_t* k_mt = keys;
  int32_t* k_r = k_mt + a.d_mt_slots;
  T* v_mt = vals;
  T* v_r = v_mt + a.d_mt_slots;
  const int b_mt = Log2(a.d_mt_slots);
  const int b_r = Log2(a.d_r_slots);
  const int r_limit = a.d_r_slots / 2;  // distinct keys of R(j, :) the table takes
  ClearWords(bm, kDropWindowWords, lane);
  ClearWords(summary, kSummary, lane);
  FusedState* state = a.state;
  const int64_t parity = state->parity;
  const int64_t other = parity ^ 1;
  const T alpha = static_cast<T>(state->alpha);
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  unsigned long long written = 0;
  int overflow = 0;
  for (int64_t j = warp; j < a.n; j += warps) {
    const int nm = a.m_cnt[j];
    const int nz = a.z_cnt[j];
    const int nmt = a.mt_cnt[parity][j];
    if (nmt > a.cap_mt) {
      overflow |= kOverflowMt;
      continue;
    }
    ClearTable(keys, table, lane);
    // M(:, j) and Z(:, j) into shared memory (sorted by row), then M(j, :) into its hash
    for (int e = lane; e < nm; e += kWarp) {
      mr[e] = a.m_rows[j * a.topk + e];
      mv[e] = a.m_vals[j * a.topk + e];
    }
    for (int e = lane; e < nz; e += kWarp) {
      zr[e] = a.z_rows[j * a.cap_z + e];
      zv[e] = a.z_vals[j * a.cap_z + e];
    }
    __syncwarp();
    const int32_t* mtc = a.mt_cols[parity] + j * a.cap_mt;
    const T* mtv = a.mt_vals[parity] + j * a.cap_mt;
    int32_t lo = static_cast<int32_t>(j);
    int32_t hi = static_cast<int32_t>(j);
    bool fresh;
    // M(:, j) and Z(:, j) are sorted: their ends bound the window, and lookups are binary searches
    if (nm > 0) {
      lo = min(lo, mr[0]);
      hi = max(hi, mr[nm - 1]);
    }
    if (nz > 0) {
      lo = min(lo, zr[0]);
      hi = max(hi, zr[nz - 1]);
    }
    for (int e = lane; e < nmt; e += kWarp) {
      const int at = FindOrInsert(k_mt, b_mt, mtc[e], &fresh);
      v_mt[at] = mtv[e];
      lo = min(lo, mtc[e]);
      hi = max(hi, mtc[e]);
    }
    // R(j, :) = e_j^T - A(j, :) M: terms in ascending k for every column i.  Lane u holds
    // entry u of row j of A and the length of row k_u of M^T; the rows of M^T are loaded
    // one step ahead of the step that adds them, so their loads overlap.
    int32_t k_lane = -1;
    T a_lane = T(0);
    int nk_lane = 0;
    if (lane < a.ell) {
      k_lane = a.a_rows_ell[j * a.ell + lane];
      if (k_lane >= 0) {
        a_lane = a.a_rows_ell_val[j * a.ell + lane];
        nk_lane = a.mt_cnt[parity][k_lane];
      }
    }
    int r_keys = 0;
    bool r_full = __any_sync(0xffffffffu, nk_lane > a.cap_mt);
    int32_t cur_i[kMtPerLane];
    T cur_v[kMtPerLane];
    int32_t next_i[kMtPerLane];
    T next_v[kMtPerLane];
    auto load_row = [&](int u, int32_t (&ii)[kMtPerLane], T (&vv)[kMtPerLane]) {
      const int32_t k = __shfl_sync(0xffffffffu, k_lane, u);
      const int nk = r_full ? 0 : __shfl_sync(0xffffffffu, nk_lane, u);
      const int32_t* kc = a.mt_cols[parity] + static_cast<int64_t>(k) * a.cap_mt;
      const T* kv = a.mt_vals[parity] + static_cast<int64_t>(k) * a.cap_mt;
#pragma unroll
      for (int q = 0; q < kMtPerLane; ++q) {
        const int e = q * kWarp + lane;
        ii[q] = -1;
        vv[q] = T(0);
        if (k >= 0 && e < nk) {
          ii[q] = kc[e];
          vv[q] = kv[e];
        }
      }
    };
    load_row(0, cur_i, cur_v);
    for (int u = 0; u < a.ell && !r_full; ++u) {
      const int32_t k = __shfl_sync(0xffffffffu, k_lane, u);
      const int nk = __shfl_sync(0xffffffffu, nk_lane, u);
      const T a_jk = __shfl_sync(0xffffffffu, a_lane, u);
      if (u + 1 < a.ell) load_row(u + 1, next_i, next_v);
      if (k >= 0) {  // warp-uniform
#pragma unroll
        for (int q = 0; q < kMtPerLane; ++q) {
          if (q * kWarp < nk) {  // warp-uniform
            const int e = q * kWarp + lane;
            bool is_new = false;
            bool lost = false;
            if (e < nk) {
              const int32_t i = cur_i[q];
              const T prod = Mul(a_jk, cur_v[q]);
              const int at = FindOrInsert(k_r, b_r, i, &is_new);
              if (at < 0) {
                lost = true;
              } else {
                // a column i appears once in row k of M: no two lanes share a slot here
                v_r[at] = is_new ? prod : Add(v_r[at], prod);
                lo = min(lo, i);
                hi = max(hi, i);
              }
            }
            r_keys += __popc(__ballot_sync(0xffffffffu, is_new));
            if (__any_sync(0xffffffffu, lost)) r_full = true;
          }
        }
        __syncwarp();
        if (r_keys > r_limit) r_full = true;
      }
#pragma unroll
      for (int q = 0; q < kMtPerLane; ++q) {
        cur_i[q] = next_i[q];
        cur_v[q] = next_v[q];
      }
    }
    if (r_full) {
      overflow |= kOverflowRow;
      continue;
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    // S(:, j) in row order, one window of kDropWindowRows rows at a time
    int count = 0;
    bool too_long = false;
    for (int32_t seg_lo = lo; seg_lo <= hi; seg_lo += kDropWindowRows) {
      const int32_t seg_hi = hi - seg_lo < kDropWindowRows ? hi : seg_lo + (kDropWindowRows - 1);
      const int words = (seg_hi - seg_lo) / 32 + 1;
      if (lane == 0 && j >= seg_lo && j <= seg_hi) MarkRow(bm, summary, static_cast<int>(j - seg_lo));
      for (int e = lane; e < nm; e += kWarp) {
        if (mr[e] >= seg_lo && mr[e] <= seg_hi) MarkRow(bm, summary, mr[e] - seg_lo);
      }
      for (int e = lane; e < nz; e += kWarp) {
        if (zr[e] >= seg_lo && zr[e] <= seg_hi) MarkRow(bm, summary, zr[e] - seg_lo);
      }
      for (int t = lane; t < table; t += kWarp) {
        const int32_t key = keys[t];
        if (key != kEmpty && key >= seg_lo && key <= seg_hi) MarkRow(bm, summary, key - seg_lo);
      }
      __syncwarp();
      const int found = DrainRows(bm, summary, SummaryWords(words), rows, lane);
      if (count + found > kDropCap || found > kDropRowsCap) {
        too_long = true;
        break;
      }
      for (int r0 = 0; r0 < found; r0 += kWarp) {
        const int r = r0 + lane;
        bool emit = false;
        int32_t i = 0;
        T v = T(0);
        if (r < found) {
          i = seg_lo + static_cast<int32_t>(rows[r]);
          // U(i, j) = M(i, j) (+) alpha Z(i, j)
          int pm = LowerBoundShared(mr, nm, i);
          int pz = LowerBoundShared(zr, nz, i);
          pm = pm < nm && mr[pm] == i ? pm : -1;
          pz = pz < nz && zr[pz] == i ? pz : -1;
          const bool own = pm >= 0 || pz >= 0;
          T u_own = T(0);
          if (pm >= 0 && pz >= 0) {
            u_own = Add(mv[pm], Mul(alpha, zv[pz]));
          } else if (pm >= 0) {
            u_own = Add(mv[pm], T(0));
          } else if (pz >= 0) {
            u_own = Add(T(0), Mul(alpha, zv[pz]));
          }
          // U(j, i) = M(j, i) (+) alpha Z(j, i), Z(j, i) = pr_j R(j, i) unless R(j, i) is an exact zero
          const int pmt = FindSlot(k_mt, b_mt, i);
          const int pr = FindSlot(k_r, b_r, i);
          bool z_row = false;
          T z_ji = T(0);
          if (pr >= 0 || static_cast<int64_t>(i) == j) {
            T rv = pr >= 0 ? -v_r[pr] : T(0);
            if (static_cast<int64_t>(i) == j) rv = Add(rv, T(1));
            if (!(rv == T(0))) {
              z_row = true;
              z_ji = Mul(a.pr[j], rv);
            }
          }
          const bool trans = pmt >= 0 || z_row;
          T u_tr = T(0);
          if (pmt >= 0 && z_row) {
            u_tr = Add(v_mt[pmt], Mul(alpha, z_ji));
          } else if (pmt >= 0) {
            u_tr = Add(v_mt[pmt], T(0));
          } else if (z_row) {
            u_tr = Add(T(0), Mul(alpha, z_ji));
          }
          // the half sum of the symmetrisation (dropping.cpp:106-120)
          if (own && trans) {
            v = Mul(T(0.5), Add(u_own, u_tr));
          } else if (own) {
            v = Mul(T(0.5), Add(u_own, T(0)));
          } else if (trans) {
            v = Mul(T(0.5), Add(T(0), u_tr));
          }
          emit = own || trans;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, emit);
        if (emit) {
          const int o = count + __popc(mask & LaneMaskBelow());
          s.keys[o] = i;
          s.vals[o] = static_cast<double>(v);
        }
        count += __popc(mask);
      }
      __syncwarp();
    }
    if (too_long) {
      // leave the bitmap clear for the next column before skipping this one
      for (int32_t seg_lo = lo; seg_lo <= hi; seg_lo += kDropWindowRows) {
        const int32_t seg_hi = hi - seg_lo < kDropWindowRows ? hi : seg_lo + (kDropWindowRows - 1);
        ClearWords(bm, (seg_hi - seg_lo) / 32 + 1, lane);
        ClearWords(summary, SummaryWords((seg_hi - seg_lo) / 32 + 1), lane);
      }
      __syncwarp();
      overflow |= kOverflowSide;
      continue;
    }
    __syncwarp();
    const int kept = DecideDrops(s, count, j, a.topk, lane);
    // survivors: M(:, j) in place, and M^T into the other set
    int32_t* out_rows = a.m_rows + j * a.topk;
    T* out_vals = a.m_vals + j * a.topk;
    int at = 0;
    for (int b0 = 0; b0 < count; b0 += kWarp) {
      const int i = b0 + lane;
      const bool keep = i < count && s.keep[i] != 0;
      const unsigned mask = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int o = at + __popc(mask & LaneMaskBelow());
        const int32_t row = s.keys[i];
        const T v = static_cast<T>(s.vals[i]);
        out_rows[o] = row;
        out_vals[o] = v;
        const int slot = atomicAdd(&a.mt_cnt[other][row], 1);
        if (slot < a.cap_mt) {
          a.mt_cols[other][static_cast<int64_t>(row) * a.cap_mt + slot] = static_cast<int32_t>(j);
          a.mt_vals[other][static_cast<int64_t>(row) * a.cap_mt + slot] = v;
        } else {
          overflow |= kOverflowMt;
        }
      }
      at += __popc(mask);
    }
    if (lane == 0) a.m_cnt[j] = kept;
    written += static_cast<unsigned long long>(kept);
    __syncwarp();
  }
  overflow = __reduce_or_sync(0xffffffffu, overflow);
  if (lane == 0) {
    if (written != 0ull) atomicAdd(&state->nnz_m, written);
    if (overflow != 0) atomicOr(&state->overflow, overflow);
  }
}

// ---------------------------------------------------------------------------
// Residual kernel: R = I - A M(:, j), Z = Pr R, ||R(:, j)||^2, then the MR
// projection of A Z(:, j).  The arithmetic is ColumnProductKernel's
// (spgemm.cu): rows in ascending order from the window bitmap, each row of A
// (ELL copy) pulled in ascending k against a hash of the column, the
// accumulator started at -0.0, sums sequential in row order on one lane.

template <class T>
__host__ __device__ size_t ResidualSlabBytes(int m_slots, int z_slots) {
  return Round16(static_cast<size_t>(kWindowWords) * 4) + Round16(static_cast<size_t>(SummaryWords(kWindowWords)) * 4) +
         Round16(static_cast<size_t>(kRowsCap) * 2) + Round16(static_cast<size_t>(m_slots) * 4) +
         Round16(static_cast<size_t>(m_slots) * sizeof(T)) + Round16(static_cast<size_t>(z_slots) * 4) +
         Round16(static_cast<size_t>(z_slots) * sizeof(T)) + 2 * Round16(kWarp * sizeof(double));
}

// Sequential sum of `count` staged values onto s (one lane).
__device__ __forceinline__ double SumStaged(double s, const double* src, int count) {
  if (count == kWarp) {
    const double2* src2 = reinterpret_cast<const double2*>(src);
#pragma unroll
    for (int l = 0; l < kWarp / 2; ++l) {
      const double2 v = src2[l];
      s = Add(s, v.x);
      s = Add(s, v.y);
    }
  } else {
    for (int l = 0; l < count; ++l) s = Add(s, src[l]);
  }
  return s;
}

template <class T, int kEll>
__global__ void __launch_bounds__(kResidualWarps * kWarp) FusedResidualKernel(FusedArgs<T> a) {
  extern __shared__ __align__(16) unsigned char fused_res_smem[];
  const int lane = threadIdx.x & 31;
  constexpr int kSummary = (kWindowWords + kWarp * kWarp - 1) / (kWarp * kWarp) * kWarp;
  unsigned char* base = fused_res_smem + (threadIdx.x >> 5) * ResidualSlabBytes<T>(a.m_hash_slots, a.z_hash_slots);
  uint32_t* bm = reinterpret_cast<uint32_t*>(base);
  base += Round16(static_cast<size_t>(kWindowWords) * 4);
  uint32_t* summary = reinterpret_cast<uint32_t*>(base);
  base += Round16(static_cast<size_t>(kSummary) * 4);
  uint16_t* rows = reinterpret_cast<uint16_t*>(base);
  base += Round16(static_cast<size_t>(kRowsCap) * 2);
  int32_t* mkeys = reinterpret_cast<int32_t*>(base);
  base += Round16(static_cast<size_t>(a.m_hash_slots) * 4);
  T* mvals = reinterpret_cast<T*>(base);
  base += Round16(static_cast<size_t>(a.m_hash_slots) * sizeof(T));
  int32_t* zkeys = reinterpret_cast<int32_t*>(base);
  base += Round16(static_cast<size_t>(a.z_hash_slots) * 4);
  T* zvals = reinterpret_cast<T*>(base);
  base += Round16(static_cast<size_t>(a.z_hash_slots) * sizeof(T));
  double* stage0 = reinterpret_cast<double*>(base);
  double* stage1 = stage0 + kWarp;
  const int mbits = Log2(a.m_hash_slots) - 1;  // buckets of two slots
  const int zbits = Log2(a.z_hash_slots) - 1;
  ClearWords(bm, kWindowWords, lane);
  ClearWords(summary, kSummary, lane);
  __syncwarp();
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  unsigned long long written = 0;
  int overflow = 0;
  const int64_t read_set = a.state->parity;  // the M^T set the drop kernel has just read
  for (int64_t j = warp; j < a.n; j += warps) {
    // ---- R(:, j) = e_j - A M(:, j) ----------------------------------------
    if (lane == 0) a.mt_cnt[read_set][j] = 0;  // that set refills from zero in the next drop kernel
    const int nm = a.m_cnt[j];
    ClearTable(mkeys, a.m_hash_slots, lane);
    __syncwarp();
    int32_t k_mine = -1;
    bool placed = true;
    if (lane < nm) {
      k_mine = a.m_rows[j * a.topk + lane];
      placed = BucketInsert(mkeys, mvals, mbits, k_mine, a.m_vals[j * a.topk + lane]);
    }
    const bool m_displaced = !__all_sync(0xffffffffu, placed);
    // the candidate rows: A(:, k) for k in M(:, j), and j itself
    int32_t cand[kEll];
    int32_t lo = static_cast<int32_t>(j);
    int32_t hi = static_cast<int32_t>(j);
#pragma unroll
    for (int u = 0; u < kEll / 4; ++u) {
      int4 r4 = make_int4(-1, -1, -1, -1);
      if (k_mine >= 0) r4 = reinterpret_cast<const int4*>(a.a_cols_ell + static_cast<int64_t>(k_mine) * kEll)[u];
      cand[4 * u] = r4.x;
      cand[4 * u + 1] = r4.y;
      cand[4 * u + 2] = r4.z;
      cand[4 * u + 3] = r4.w;
    }
#pragma unroll
    for (int u = 0; u < kEll; ++u) {
      if (cand[u] >= 0) {
        lo = min(lo, cand[u]);
        hi = max(hi, cand[u]);
      }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    int32_t* zr_out = a.z_rows + j * a.cap_z;
    T* zv_out = a.z_vals + j * a.cap_z;
    ClearTable(zkeys, a.z_hash_slots, lane);
    __syncwarp();
    int kept = 0;
    double sq = 0.0;
    bool z_placed = true;
    // the rows in ascending order, one window of kWindowRows rows at a time
    for (int32_t seg_lo = lo; seg_lo <= hi; seg_lo += kWindowRows) {
      const int32_t seg_hi = hi - seg_lo < kWindowRows ? hi : seg_lo + (kWindowRows - 1);
      const int words = (seg_hi - seg_lo) / 32 + 1;
      if (lane == 0 && j >= seg_lo && j <= seg_hi) MarkRow(bm, summary, static_cast<int>(j - seg_lo));
#pragma unroll
      for (int u = 0; u < kEll; ++u) {
        if (cand[u] >= seg_lo && cand[u] <= seg_hi) MarkRow(bm, summary, cand[u] - seg_lo);
      }
      __syncwarp();
      const int count = DrainRows(bm, summary, SummaryWords(words), rows, lane);
      for (int r0 = 0; r0 < count; r0 += kWarp) {
        const int r = r0 + lane;
        bool keep = false;
        int32_t i = 0;
        T v = T(0);
        if (r < count) {
          i = seg_lo + static_cast<int32_t>(rows[r]);
          T acc = T(-0.0);
          const int4* ks = reinterpret_cast<const int4*>(a.a_rows_ell + static_cast<int64_t>(i) * kEll);
          const T* vs = a.a_rows_ell_val + static_cast<int64_t>(i) * kEll;
#pragma unroll
          for (int u = 0; u < kEll / 4; ++u) {
            const int4 k4 = ks[u];
            T v4[4];
            LoadFour(vs + 4 * u, v4);
            const int32_t kk[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              T bv;
              if (kk[e] >= 0 && BucketFind(mkeys, mvals, mbits, m_displaced, kk[e], bv)) acc = Add(acc, Mul(v4[e], bv));
            }
          }
          v = -acc;
          if (static_cast<int64_t>(i) == j) v = Add(v, T(1));
          const double sd = static_cast<double>(v);
          stage0[lane] = Mul(sd, sd);
          keep = !(v == T(0));  // Eigen prune(0.0)
        }
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const int o = kept + __popc(mask & LaneMaskBelow());
          const T z = Mul(a.pr[i], v);
          zr_out[o] = i;
          zv_out[o] = z;
          z_placed &= BucketInsert(zkeys, zvals, zbits, i, z);
        }
        kept += __popc(mask);
        __syncwarp();
        if (lane == 0) sq = SumStaged(sq, stage0, min(kWarp, count - r0));
        __syncwarp();
      }
    }
    if (lane == 0) {
      a.sq[j] = sq;
      a.z_cnt[j] = kept;
    }
    written += static_cast<unsigned long long>(kept);
    const bool z_displaced = !__all_sync(0xffffffffu, z_placed);
    // ---- projection: tt = ||Pr A Z(:, j)||^2, bt = <Z(:, j), Pr A Z(:, j)> --
    lo = INT32_MAX;
    hi = -1;
    for (int e = lane; e < kept; e += kWarp) {
      const int4* src = reinterpret_cast<const int4*>(a.a_cols_ell + static_cast<int64_t>(zr_out[e]) * kEll);
#pragma unroll
      for (int u = 0; u < kEll / 4; ++u) {
        const int4 r4 = src[u];
        const int32_t rr[4] = {r4.x, r4.y, r4.z, r4.w};
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          if (rr[t] >= 0) {
            lo = min(lo, rr[t]);
            hi = max(hi, rr[t]);
          }
        }
      }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    double proj = 0.0;  // tt on lane 0, bt on lane 1
    for (int32_t seg_lo = lo; seg_lo <= hi; seg_lo += kWindowRows) {
      const int32_t seg_hi = hi - seg_lo < kWindowRows ? hi : seg_lo + (kWindowRows - 1);
      const int words2 = (seg_hi - seg_lo) / 32 + 1;
      for (int e = lane; e < kept; e += kWarp) {
        const int4* src = reinterpret_cast<const int4*>(a.a_cols_ell + static_cast<int64_t>(zr_out[e]) * kEll);
#pragma unroll
        for (int u = 0; u < kEll / 4; ++u) {
          const int4 r4 = src[u];
          const int32_t rr[4] = {r4.x, r4.y, r4.z, r4.w};
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            if (rr[t] >= seg_lo && rr[t] <= seg_hi) MarkRow(bm, summary, rr[t] - seg_lo);
          }
        }
      }
      __syncwarp();
      const int count2 = DrainRows(bm, summary, SummaryWords(words2), rows, lane);
      for (int r0 = 0; r0 < count2; r0 += kWarp) {
        const int r = r0 + lane;
        if (r < count2) {
          const int32_t i = seg_lo + static_cast<int32_t>(rows[r]);
          T acc = T(-0.0);
          const int4* ks = reinterpret_cast<const int4*>(a.a_rows_ell + static_cast<int64_t>(i) * kEll);
          const T* vs = a.a_rows_ell_val + static_cast<int64_t>(i) * kEll;
#pragma unroll
          for (int u = 0; u < kEll / 4; ++u) {
            const int4 k4 = ks[u];
            T v4[4];
            LoadFour(vs + 4 * u, v4);
            const int32_t kk[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              T bv;
              if (kk[e] >= 0 && BucketFind(zkeys, zvals, zbits, z_displaced, kk[e], bv)) acc = Add(acc, Mul(v4[e], bv));
            }
          }
          const double td = static_cast<double>(Mul(a.pr[i], acc));
          T zi;
          stage0[lane] = Mul(td, td);
          // rows of Z absent from the product add +0.0, which leaves a sum started at +0.0 unchanged
          stage1[lane] = BucketFind(zkeys, zvals, zbits, z_displaced, i, zi) ? Mul(static_cast<double>(zi), td) : 0.0;
        }
        __syncwarp();
        // lane 0 extends tt and lane 1 bt, side by side in one instruction stream
        const int span = min(kWarp, count2 - r0);
        if (lane < 2) proj = SumStaged(proj, lane == 0 ? stage0 : stage1, span);
        __syncwarp();
      }
    }
    if (lane == 0) a.tt[j] = proj;
    if (lane == 1) a.bt[j] = proj;
    __syncwarp();
  }
  overflow = __reduce_or_sync(0xffffffffu, overflow);
  if (lane == 0) {
    if (written != 0ull) atomicAdd(&a.state->nnz_z, written);
    if (overflow != 0) atomicOr(&a.state->overflow, overflow);
  }
}

// ---------------------------------------------------------------------------
// Decide kernel: the three tree sums; the last block appends the history row,
// applies the stop rules (result_operations.cpp:53-67, minimal_residual.cpp:55-89),
// forms the next step length and, inside the graph, sets the loop condition.
template <class T>
__global__ void __launch_bounds__(kTreeLanes) FusedDecideKernel(FusedArgs<T> a, cudaGraphConditionalHandle loop,
                                                                bool in_graph) {
  __shared__ double shared[kTreeLanes];
  __shared__ int last;
  const int t = threadIdx.x;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTreeChunk + t;
  double s_sq = 0.0;
  double s_bt = 0.0;
  double s_tt = 0.0;
#pragma unroll
  for (int m = 0; m < kTreeTerms; ++m) {
    const int64_t i = base + static_cast<int64_t>(kTreeLanes) * m;
    if (i < a.n) {
      s_sq = Add(s_sq, a.sq[i]);
      s_bt = Add(s_bt, a.bt[i]);
      s_tt = Add(s_tt, a.tt[i]);
    }
  }
  double total_sq = TreeButterfly(s_sq, shared);
  double total_bt = TreeButterfly(s_bt, shared);
  double total_tt = TreeButterfly(s_tt, shared);
  FusedState* state = a.state;
  if (gridDim.x > 1) {
    const int64_t chunks = gridDim.x;
    if (t == 0) {
      a.chunk[blockIdx.x] = total_sq;
      a.chunk[chunks + blockIdx.x] = total_bt;
      a.chunk[2 * chunks + blockIdx.x] = total_tt;
      __threadfence();
      last = atomicAdd(&state->arrive, 1u) == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    total_sq = TreeLevel(a.chunk, chunks, shared);
    total_bt = TreeLevel(a.chunk + chunks, chunks, shared);
    total_tt = TreeLevel(a.chunk + 2 * chunks, chunks, shared);
  }
  if (t != 0) return;
  state->arrive = 0u;
  const int64_t it = state->iteration + 1;
  const double entries = Mul(static_cast<double>(a.n), static_cast<double>(a.n));
  FusedRow row;
  row.iteration = it;
  row.residual_norm = __dsqrt_rn(total_sq);
  row.density_m = __ddiv_rn(static_cast<double>(state->nnz_m), entries);
  // the row's direction is the Z the step M += alpha Z used, not the one just formed
  // (the history row is appended before Z is recomputed, minimal_residual.cpp:78-88)
  row.density_direction = __ddiv_rn(static_cast<double>(state->nnz_dir), entries);
  a.history[it] = row;
  state->iteration = it;
  state->last_nnz_m = state->nnz_m;
  state->last_nnz_z = state->nnz_z;
  state->nnz_dir = state->nnz_z;
  state->nnz_m = 0ull;
  state->nnz_z = 0ull;
  int stop = kRunning;
  if (state->overflow != 0) {
    stop = kOverflowStop;
  } else if (row.residual_norm < a.tolerance) {
    stop = kConverged;
  } else if (it >= a.max_iterations) {
    stop = kIterationLimit;
  } else {
    // the next iteration's step length (minimal_residual.cpp:55-60)
    const double num = total_bt;
    const double den = total_tt;
    if (!isfinite(den) || !(fabs(den) > 0.0)) {
      stop = kBreakdown;
    } else {
      const double alpha = __ddiv_rn(num, den);
      if (!isfinite(alpha)) {
        stop = kBreakdown;
      } else {
        state->alpha = alpha;
      }
    }
  }
  state->stop = stop;
  state->parity ^= 1;
  state->bodies += 1;
  if (in_graph) {
    // the body count bounds the loop whatever the recurrence does
    const bool again = stop == kRunning && state->bodies < a.max_iterations + 1;
    cudaGraphSetConditional(loop, again ? 1u : 0u);
  }
}

// ---------------------------------------------------------------------------
// Conversions between compact CSC and the slots.

// Column j of a compact CSC into `cap` slots (count per column); when t_cnt is
// given, every entry (i, j) is also appended to row i of the transposed slots.
template <class T>
__global__ void ToSlotsKernel(CscView<T> x, int cap, int32_t* __restrict__ rows, T* __restrict__ vals,
                              int32_t* __restrict__ cnt, int t_cap, int32_t* __restrict__ t_cols, T* __restrict__ t_vals,
                              int32_t* __restrict__ t_cnt, FusedState* __restrict__ state) {
  int overflow = 0;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < x.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = x.ptr[j];
    const int64_t e = x.ptr[j + 1];
    const int len = static_cast<int>(e - b);
    if (len > cap) {
      overflow |= kOverflowSide;
      cnt[j] = 0;
      continue;
    }
    for (int q = 0; q < len; ++q) {
      const int32_t i = x.idx[b + q];
      const T v = x.val[b + q];
      rows[j * cap + q] = i;
      vals[j * cap + q] = v;
      if (t_cnt != nullptr) {
        const int slot = atomicAdd(&t_cnt[i], 1);
        if (slot < t_cap) {
          t_cols[static_cast<int64_t>(i) * t_cap + slot] = static_cast<int32_t>(j);
          t_vals[static_cast<int64_t>(i) * t_cap + slot] = v;
        } else {
          overflow |= kOverflowMt;
        }
      }
    }
    cnt[j] = len;
  }
  if (overflow != 0) atomicOr(&state->overflow, overflow);
}

__global__ void WidenCountsKernel(const int32_t* __restrict__ cnt, int64_t n, int64_t* __restrict__ out) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[j] = cnt[j];
  }
}

template <class T>
__global__ void FromSlotsKernel(int64_t n, int cap, const int32_t* __restrict__ rows, const T* __restrict__ vals,
                                const int64_t* __restrict__ ptr, int32_t* __restrict__ idx_out, T* __restrict__ val_out) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t o = ptr[j];
    const int len = static_cast<int>(ptr[j + 1] - o);
    for (int q = 0; q < len; ++q) {
      idx_out[o + q] = rows[j * cap + q];
      val_out[o + q] = vals[j * cap + q];
    }
  }
}

int CapZ(const FusedMrProblem& p) {
  const int64_t bound = 1 + static_cast<int64_t>(p.topk) * p.a_longest;
  return static_cast<int>(std::min<int64_t>(p.n, bound));
}

int NextPow2Int(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

int CapMt(const FusedMrProblem& p) { return static_cast<int>(std::min<int64_t>(p.n, 4 * static_cast<int64_t>(p.topk))); }

// Slots of the drop kernel's hash of R(j, :): twice the row's bound (every entry of row j of A times a row of M)
// up to 256; a longer row flags an overflow.
int DropRowSlots(const FusedMrProblem& p) {
  const int64_t bound = static_cast<int64_t>(p.a_longest) * CapMt(p) + 1;
  return NextPow2Int(static_cast<int>(std::min<int64_t>(std::max<int64_t>(2 * bound, kWarp), 256)));
}

std::atomic<bool> g_fused_mr_enabled{true};

template <class T>
class FusedMr final : public FusedMrBase {
 public:
  ~FusedMr() override {
    if (exec_ != nullptr) cudaGraphExecDestroy(exec_);
  }

  FusedMrOutcome Run(Ctx& ctx, const FusedMrProblem& problem, void* m_csc, const void* z_csc, double alpha,
                     std::vector<SingleIterationData>& history) override {
    FusedMrOutcome outcome;
    if (!FusedMrApplicable(problem)) return outcome;
    auto& m = *static_cast<DevCsc<T>*>(m_csc);
    const auto& z = *static_cast<const DevCsc<T>*>(z_csc);
    const int64_t n = problem.n;
    Reserve(ctx, problem);
    Configure(problem);
    const cudaStream_t st = ctx.stream;
    // state: iteration 0 is in the history; M^T set 0 is filled below
    FusedState init{};
    init.alpha = alpha;
    init.nnz_dir = static_cast<unsigned long long>(z.nnz);
    *host_state_ = init;
    SPAI_CUDA(cudaMemcpyAsync(state_.data(), host_state_, sizeof(FusedState), cudaMemcpyHostToDevice, st));
    for (int s = 0; s < 2; ++s) SPAI_CUDA(cudaMemsetAsync(mt_cnt_[s].data(), 0, sizeof(int32_t) * n, st));
    const int grid = GridFor(n, 128);
    ToSlotsKernel<T><<<grid, 128, 0, st>>>(View(m), args_.topk, args_.m_rows, args_.m_vals, args_.m_cnt, args_.cap_mt,
                                           args_.mt_cols[0], args_.mt_vals[0], args_.mt_cnt[0], args_.state);
    SPAI_LAUNCH_CHECK();
    ToSlotsKernel<T><<<grid, 128, 0, st>>>(View(z), args_.cap_z, args_.z_rows, args_.z_vals, args_.z_cnt, 0,
                                           nullptr, nullptr, nullptr, args_.state);
    SPAI_LAUNCH_CHECK();
    FusedState out;
    if (prof::Enabled()) {
      out = RunStepwise(ctx, problem, m.nnz, z.nnz);
    } else {
      if (exec_ == nullptr) Capture();
      {
        prof::Scope scope(st, "fused_mr_loop", 0.0);
        SPAI_CUDA(cudaGraphLaunch(exec_, st));
      }
      SPAI_CUDA(cudaMemcpyAsync(host_state_, state_.data(), sizeof(FusedState), cudaMemcpyDeviceToHost, st));
      ctx.Sync();
      out = *host_state_;
      CountLaunches(3 * out.bodies);
    }
    outcome.ran = true;
    outcome.graph_bodies = out.bodies;
    if (out.stop == kOverflowStop || out.overflow != 0) {
      outcome.overflow = true;
      return outcome;
    }
    const int64_t rows = out.iteration;
    std::vector<FusedRow> host_rows(static_cast<size_t>(rows + 1));
    SPAI_CUDA(cudaMemcpyAsync(host_rows.data(), args_.history, sizeof(FusedRow) * (rows + 1), cudaMemcpyDeviceToHost,
                              st));
    // M back to compact CSC
    DevCsc<T> result;
    result.Shape(n, n, st);
    ctx.counts.Reserve(static_cast<size_t>(n + 1), st);
    WidenCountsKernel<<<GridFor(n, 256), 256, 0, st>>>(args_.m_cnt, n, ctx.counts.data());
    SPAI_LAUNCH_CHECK();
    const int64_t nnz = ScanCounts(ctx, ctx.counts.data(), n, result.ptr.data());
    result.ReserveNnz(nnz, st);
    FromSlotsKernel<T><<<grid, 128, 0, st>>>(n, args_.topk, args_.m_rows, args_.m_vals, result.ptr.data(),
                                             result.idx.data(), result.val.data());
    SPAI_LAUNCH_CHECK();
    m.Swap(result);
    ctx.Sync();
    for (int64_t r = 1; r <= rows; ++r) {
      SingleIterationData row;
      row.iteration = host_rows[r].iteration;
      row.residual_norm = host_rows[r].residual_norm;
      row.density_m = host_rows[r].density_m;
      row.density_direction = host_rows[r].density_direction;
      history.push_back(row);
    }
    outcome.iterations = rows;
    outcome.converged = out.stop == kConverged;
    return outcome;
  }

 private:
  // The same three kernels launched one by one with the library's CUDA-event
  // accounting around each (spai_profile_enable): the decide kernel's result
  // is read back after every iteration, in place of the graph's condition.
  FusedState RunStepwise(Ctx& ctx, const FusedMrProblem& p, int64_t m_nnz, int64_t z_nnz) {
    const cudaStream_t st = ctx.stream;
    const double e = static_cast<double>(sizeof(T) + sizeof(int32_t));
    const double n = static_cast<double>(p.n);
    const double a_bytes = static_cast<double>(p.a_nnz) * e + 8.0 * (n + 1.0);
    double m_prev = static_cast<double>(m_nnz);
    double z_prev = static_cast<double>(z_nnz);
    FusedState out{};
    for (int64_t body = 0; body <= p.max_iterations; ++body) {
      {
        prof::Scope scope(st, "fused_drop", 0.0);
        FusedDropKernel<T><<<drop_grid_, kDropWarps * kWarp, drop_smem_, st>>>(args_);
        SPAI_LAUNCH_CHECK();
      }
      {
        prof::Scope scope(st, "fused_residual", 0.0);
        res_kernel_<<<res_grid_, kResidualWarps * kWarp, res_smem_, st>>>(args_);
        SPAI_LAUNCH_CHECK();
      }
      {
        prof::Scope scope(st, "fused_decide", 24.0 * n);
        FusedDecideKernel<T><<<decide_grid_, kTreeLanes, 0, st>>>(args_, 0, false);
        SPAI_LAUNCH_CHECK();
      }
      SPAI_CUDA(cudaMemcpyAsync(host_state_, state_.data(), sizeof(FusedState), cudaMemcpyDeviceToHost, st));
      ctx.Sync();
      out = *host_state_;
      // algorithmic bytes: the drop step reads M, Z and both transposes and writes M and M^T; the
      // residual step reads M, A and Pr, writes Z, Z^T and the three column sums
      const double m_new = static_cast<double>(out.last_nnz_m);
      const double z_new = static_cast<double>(out.last_nnz_z);
      prof::AddBytes("fused_drop", e * (2.0 * m_prev + 2.0 * z_prev + 2.0 * m_new) + 4.0 * 6.0 * n);
      prof::AddBytes("fused_residual",
                     e * m_new + a_bytes + sizeof(T) * n + 2.0 * e * z_new + 4.0 * 3.0 * n + 24.0 * n);
      m_prev = m_new;
      z_prev = z_new;
      if (out.stop != kRunning) break;
    }
    return out;
  }

  void Reserve(Ctx& ctx, const FusedMrProblem& p) {
    const cudaStream_t st = ctx.stream;
    const int64_t n = p.n;
    const int cap_z = CapZ(p);
    const int cap_mt = CapMt(p);
    const size_t un = static_cast<size_t>(n);
    m_rows_.Reserve(un * p.topk, st);
    m_vals_.Reserve(un * p.topk, st);
    m_cnt_.Reserve(un, st);
    for (int s = 0; s < 2; ++s) {
      mt_cols_[s].Reserve(un * cap_mt, st);
      mt_vals_[s].Reserve(un * cap_mt, st);
      mt_cnt_[s].Reserve(un, st);
    }
    z_rows_.Reserve(un * cap_z, st);
    z_vals_.Reserve(un * cap_z, st);
    z_cnt_.Reserve(un, st);
    sq_.Reserve(un, st);
    tt_.Reserve(un, st);
    bt_.Reserve(un, st);
    chunk_.Reserve(static_cast<size_t>(3 * CeilDiv(n, kTreeChunk)), st);
    history_.Reserve(static_cast<size_t>(p.max_iterations + 1), st);
    state_.Reserve(1, st);
    if (host_state_ == nullptr) {
      SPAI_CUDA(cudaMallocHost(reinterpret_cast<void**>(&host_state_), sizeof(FusedState)));
      host_state_holder_.reset(host_state_);
    }
    FusedArgs<T> a{};
    a.n = n;
    a.topk = p.topk;
    a.cap_z = cap_z;
    a.cap_mt = cap_mt;
    a.ell = p.ell_width;
    a.m_hash_slots = NextPow2Int(std::max(4 * p.topk, kWarp));
    a.z_hash_slots = NextPow2Int(std::max(2 * cap_z, kWarp));
    a.d_mt_slots = NextPow2Int(std::max(2 * cap_mt, kWarp));
    a.d_r_slots = DropRowSlots(p);
    a.max_iterations = p.max_iterations;
    a.tolerance = p.tolerance;
    a.a_cols_ell = p.a_cols_ell;
    a.a_rows_ell = p.a_rows_ell;
    a.a_rows_ell_val = static_cast<const T*>(p.a_rows_ell_val);
    a.pr = static_cast<const T*>(p.pr);
    a.m_rows = m_rows_.data();
    a.m_vals = m_vals_.data();
    a.m_cnt = m_cnt_.data();
    for (int s = 0; s < 2; ++s) {
      a.mt_cols[s] = mt_cols_[s].data();
      a.mt_vals[s] = mt_vals_[s].data();
      a.mt_cnt[s] = mt_cnt_[s].data();
    }
    a.z_rows = z_rows_.data();
    a.z_vals = z_vals_.data();
    a.z_cnt = z_cnt_.data();
    a.sq = sq_.data();
    a.tt = tt_.data();
    a.bt = bt_.data();
    a.chunk = chunk_.data();
    a.history = history_.data();
    a.state = state_.data();
    // a captured graph holds the old pointers and sizes: capture again on any change
    if (exec_ != nullptr && !SameArgs(a, args_)) {
      cudaGraphExecDestroy(exec_);
      exec_ = nullptr;
    }
    args_ = a;
  }

  static bool SameArgs(const FusedArgs<T>& x, const FusedArgs<T>& y) {
    bool same = x.n == y.n && x.topk == y.topk && x.cap_z == y.cap_z && x.cap_mt == y.cap_mt &&
                x.ell == y.ell && x.m_hash_slots == y.m_hash_slots && x.d_r_slots == y.d_r_slots &&
                x.d_mt_slots == y.d_mt_slots &&
                x.z_hash_slots == y.z_hash_slots && x.max_iterations == y.max_iterations &&
                x.tolerance == y.tolerance && x.a_cols_ell == y.a_cols_ell && x.a_rows_ell == y.a_rows_ell &&
                x.a_rows_ell_val == y.a_rows_ell_val && x.pr == y.pr && x.m_rows == y.m_rows &&
                x.m_vals == y.m_vals && x.m_cnt == y.m_cnt && x.z_rows == y.z_rows && x.z_vals == y.z_vals &&
                x.z_cnt == y.z_cnt &&
                x.sq == y.sq && x.tt == y.tt && x.bt == y.bt && x.chunk == y.chunk && x.history == y.history &&
                x.state == y.state;
    for (int s = 0; s < 2; ++s) {
      same = same && x.mt_cols[s] == y.mt_cols[s] && x.mt_vals[s] == y.mt_vals[s] && x.mt_cnt[s] == y.mt_cnt[s];
    }
    return same;
  }

  // Kernel choice, shared memory and grids (once per problem shape).
  void Configure(const FusedMrProblem& p) {
    switch (p.ell_width) {
      case 4: res_kernel_ = FusedResidualKernel<T, 4>; break;
      case 8: res_kernel_ = FusedResidualKernel<T, 8>; break;
      case 12: res_kernel_ = FusedResidualKernel<T, 12>; break;
      case 16: res_kernel_ = FusedResidualKernel<T, 16>; break;
      default: throw std::invalid_argument("fused MR: unsupported ELL width");
    }
    drop_smem_ = static_cast<size_t>(kDropWarps) *
                 DropWarpBytes<T>(args_.topk + args_.cap_z, args_.d_mt_slots, args_.d_r_slots);
    res_smem_ = static_cast<size_t>(kResidualWarps) * ResidualSlabBytes<T>(args_.m_hash_slots, args_.z_hash_slots);
    SPAI_CUDA(cudaFuncSetAttribute(FusedDropKernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(drop_smem_)));
    SPAI_CUDA(cudaFuncSetAttribute(res_kernel_, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(res_smem_)));
    int drop_blocks = 0;
    int res_blocks = 0;
    SPAI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&drop_blocks, FusedDropKernel<T>, kDropWarps * kWarp,
                                                            drop_smem_));
    SPAI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&res_blocks, res_kernel_, kResidualWarps * kWarp,
                                                            res_smem_));
    if (drop_blocks < 1 || res_blocks < 1) throw std::runtime_error("fused MR: kernels do not fit on an SM");
    int device = 0;
    SPAI_CUDA(cudaGetDevice(&device));
    int sms = 0;
    SPAI_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    drop_grid_ = static_cast<unsigned>(std::min<int64_t>(CeilDiv(args_.n, kDropWarps), int64_t{sms} * drop_blocks));
    res_grid_ =
        static_cast<unsigned>(std::min<int64_t>(CeilDiv(args_.n, kResidualWarps), int64_t{sms} * res_blocks));
    decide_grid_ = static_cast<unsigned>(CeilDiv(args_.n, kTreeChunk));
  }

  void Capture() {
    const FusedArgs<T> a = args_;
    cudaStream_t cs = nullptr;
    cudaStream_t bs = nullptr;
    cudaGraph_t graph = nullptr;
    SPAI_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    try {
      SPAI_CUDA(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
      SPAI_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      cudaStreamCaptureStatus status;
      cudaGraph_t capture_graph = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t num_deps = 0;
      SPAI_CUDA(cudaStreamGetCaptureInfo(cs, &status, nullptr, &capture_graph, &deps, &num_deps));
      cudaGraphConditionalHandle loop;
      SPAI_CUDA(cudaGraphConditionalHandleCreate(&loop, capture_graph, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams params = {};
      params.type = cudaGraphNodeTypeConditional;
      params.conditional.handle = loop;
      params.conditional.type = cudaGraphCondTypeWhile;
      params.conditional.size = 1;
      cudaGraphNode_t loop_node;
      SPAI_CUDA(cudaGraphAddNode(&loop_node, capture_graph, deps, num_deps, &params));
      SPAI_CUDA(cudaStreamUpdateCaptureDependencies(cs, &loop_node, 1, cudaStreamSetCaptureDependencies));
      cudaGraph_t body = params.conditional.phGraph_out[0];
      SPAI_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      FusedDropKernel<T><<<drop_grid_, kDropWarps * kWarp, drop_smem_, bs>>>(a);
      res_kernel_<<<res_grid_, kResidualWarps * kWarp, res_smem_, bs>>>(a);
      FusedDecideKernel<T><<<decide_grid_, kTreeLanes, 0, bs>>>(a, loop, true);
      SPAI_CUDA(cudaGetLastError());
      cudaGraph_t body_out = nullptr;
      SPAI_CUDA(cudaStreamEndCapture(bs, &body_out));
      SPAI_CUDA(cudaStreamEndCapture(cs, &graph));
      SPAI_CUDA(cudaGraphInstantiate(&exec_, graph, 0));
    } catch (...) {
      cudaStreamCaptureStatus st;
      for (cudaStream_t stream : {bs, cs}) {
        if (stream != nullptr && cudaStreamIsCapturing(stream, &st) == cudaSuccess &&
            st != cudaStreamCaptureStatusNone) {
          cudaGraph_t dropped = nullptr;
          cudaStreamEndCapture(stream, &dropped);
          if (dropped != nullptr && stream == cs) cudaGraphDestroy(dropped);
        }
      }
      if (graph != nullptr) cudaGraphDestroy(graph);
      if (bs != nullptr) cudaStreamDestroy(bs);
      cudaStreamDestroy(cs);
      cudaGetLastError();
      exec_ = nullptr;
      throw;
    }
    cudaGraphDestroy(graph);
    cudaStreamDestroy(bs);
    cudaStreamDestroy(cs);
  }

  struct PinnedFree {
    void operator()(FusedState* p) const { cudaFreeHost(p); }
  };

  DevBuf<int32_t> m_rows_, m_cnt_, z_rows_, z_cnt_;
  DevBuf<T> m_vals_, z_vals_;
  DevBuf<int32_t> mt_cols_[2], mt_cnt_[2];
  DevBuf<T> mt_vals_[2];
  DevBuf<double> sq_, tt_, bt_, chunk_;
  DevBuf<FusedRow> history_;
  DevBuf<FusedState> state_;
  FusedState* host_state_ = nullptr;
  std::unique_ptr<FusedState, PinnedFree> host_state_holder_;
  FusedArgs<T> args_{};
  cudaGraphExec_t exec_ = nullptr;
  void (*res_kernel_)(FusedArgs<T>) = nullptr;
  size_t drop_smem_ = 0;
  size_t res_smem_ = 0;
  unsigned drop_grid_ = 1;
  unsigned res_grid_ = 1;
  unsigned decide_grid_ = 1;
};

}  // namespace

bool FusedMrEnabled() { return g_fused_mr_enabled.load(std::memory_order_relaxed); }
void SetFusedMrEnabled(bool enabled) { g_fused_mr_enabled.store(enabled, std::memory_order_relaxed); }

bool FusedMrApplicable(const FusedMrProblem& p) {
  if (p.n <= 0 || p.n > kTreeChunk * kTreeChunk) return false;
  if (p.topk <= 0 || p.topk > kMaxTopK) return false;
  if (p.ell_width != 4 && p.ell_width != 8 && p.ell_width != 12 && p.ell_width != 16) return false;
  if (p.a_longest <= 0 || p.a_longest > p.ell_width) return false;
  if (p.max_iterations < 1) return false;
  const int cap_z = CapZ(p);
  // a drop column's candidate rows and a product column's row lists must fit
  const int64_t drop_candidates = p.topk + cap_z + CapMt(p) + DropRowSlots(p) / 2 + 1;
  if (drop_candidates > kDropRowsCap) return false;
  if (static_cast<int64_t>(cap_z) * p.a_longest > kRowsCap) return false;
  return true;
}

template <class T>
std::unique_ptr<FusedMrBase> MakeFusedMr() {
  return std::unique_ptr<FusedMrBase>(new FusedMr<T>());
}

template std::unique_ptr<FusedMrBase> MakeFusedMr<double>();
template std::unique_ptr<FusedMrBase> MakeFusedMr<float>();

}  // namespace spai
