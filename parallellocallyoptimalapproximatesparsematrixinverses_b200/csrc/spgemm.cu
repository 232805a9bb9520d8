// SpGEMM kernels (sm_100a).  One warp owns one output column.
//
//  symbolic : the rows of X(:,k) for every k in B(:,j) are flattened across
//             the 32 lanes and inserted into a per-warp open-addressing hash
//             in shared memory; the number of new keys is the column count.
//  numeric  : the row set is rebuilt, compacted and bitonic-sorted in shared
//             memory; column j of B is put in a second hash (k -> value); lane
//             s then computes output entry s by walking row i of X (CSR) in
//             ascending k and looking each k up in the B hash.
//
// Columns are binned by the shared memory they need (hash tables sized at
// twice the number of keys); columns beyond the largest bin use the same
// code on a global-memory workspace.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device.cuh"
#include "ops.cuh"
#include "profile.cuh"
#include "spgemm.cuh"

namespace spai {

namespace {

constexpr int32_t kEmpty = -1;

__device__ __forceinline__ unsigned LaneMaskBelow() {
  unsigned mask;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(mask));
  return mask;
}

__device__ __forceinline__ uint32_t Slot(int32_t key, int bits) {
  return (static_cast<uint32_t>(key) * 2654435761u) >> (32 - bits);
}

__host__ __device__ inline int Log2(int v) {
  int b = 0;
  while ((1 << b) < v) ++b;
  return b;
}

// Per-warp workspace (shared memory or global memory).
template <class T>
struct Space {
  double* stage0;    // slots/2
  double* stage1;    // slots/2
  T* bvals;          // slots/2
  int64_t* xstart;   // 32
  int32_t* keys;     // slots
  int32_t* sorted;   // slots/2
  int32_t* bkeys;    // slots/2
  int32_t* prefix;   // 33
  uint8_t* present;  // slots/2
};

__host__ __device__ inline size_t Round16(size_t v) { return (v + 15) & ~static_cast<size_t>(15); }

template <class T>
__host__ __device__ inline size_t SpaceBytes(int slots, bool numeric) {
  if (!numeric) {
    return Round16(32 * sizeof(int64_t)) + Round16(static_cast<size_t>(slots) * 4) + Round16(33 * 4);
  }
  const size_t half = static_cast<size_t>(slots) / 2;
  return Round16(half * 8) * 2 + Round16(half * sizeof(T)) + Round16(32 * sizeof(int64_t)) +
         Round16(static_cast<size_t>(slots) * 4) + Round16(half * 4) * 2 + Round16(33 * 4) + Round16(half);
}

template <class T>
__device__ inline Space<T> CarveSpace(unsigned char* base, int slots, bool numeric) {
  Space<T> s{};
  const size_t half = static_cast<size_t>(slots) / 2;
  if (numeric) {
    s.stage0 = reinterpret_cast<double*>(base);
    base += Round16(half * 8);
    s.stage1 = reinterpret_cast<double*>(base);
    base += Round16(half * 8);
    s.bvals = reinterpret_cast<T*>(base);
    base += Round16(half * sizeof(T));
  }
  s.xstart = reinterpret_cast<int64_t*>(base);
  base += Round16(32 * sizeof(int64_t));
  s.keys = reinterpret_cast<int32_t*>(base);
  base += Round16(static_cast<size_t>(slots) * 4);
  if (numeric) {
    s.sorted = reinterpret_cast<int32_t*>(base);
    base += Round16(half * 4);
    s.bkeys = reinterpret_cast<int32_t*>(base);
    base += Round16(half * 4);
  }
  s.prefix = reinterpret_cast<int32_t*>(base);
  base += Round16(33 * 4);
  if (numeric) {
    s.present = reinterpret_cast<uint8_t*>(base);
  }
  return s;
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

// Keys are unique: claims a slot and returns it.
__device__ __forceinline__ uint32_t ClaimSlot(int32_t* table, int bits, int32_t key) {
  const uint32_t mask = (1u << bits) - 1u;
  uint32_t h = Slot(key, bits);
  while (true) {
    const int32_t old = atomicCAS(&table[h], kEmpty, key);
    if (old == kEmpty || old == key) return h;
    h = (h + 1u) & mask;
  }
}

template <class T>
__device__ __forceinline__ bool Lookup(const int32_t* table, const T* vals, int bits, int32_t key, T& out) {
  const uint32_t mask = (1u << bits) - 1u;
  uint32_t h = Slot(key, bits);
  while (true) {
    const int32_t cur = table[h];
    if (cur == key) {
      out = vals[h];
      return true;
    }
    if (cur == kEmpty) return false;
    h = (h + 1u) & mask;
  }
}

__device__ inline void ClearTable(int32_t* table, int size, int lane) {
  for (int i = lane; i < size; i += kWarp) table[i] = kEmpty;
}

// Inserts every row of X(:,k), k in B(:,col), plus the diagonal when asked;
// returns the number of new keys (warp-uniform).
template <class T>
__device__ int InsertColumnRows(const CscView<T>& x, const CscView<T>& b, int64_t col, bool add_diag,
                                const Space<T>& s, int bits, int lane) {
  int added = 0;
  if (add_diag) {
    bool fresh = false;
    if (lane == 0) fresh = InsertKey(s.keys, bits, static_cast<int32_t>(col));
    added += __popc(__ballot_sync(0xffffffffu, fresh));
  }
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
    s.prefix[lane] = inclusive - len;
    s.xstart[lane] = xs;
    __syncwarp();
    for (int e0 = 0; e0 < total; e0 += kWarp) {
      const int e = e0 + lane;
      bool fresh = false;
      if (e < total) {
        // largest entry b with prefix[b] <= e
        int lo = 0;
        int hi = 31;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s.prefix[mid] <= e) {
            lo = mid;
          } else {
            hi = mid - 1;
          }
        }
        const int64_t q = s.xstart[lo] + (e - s.prefix[lo]);
        fresh = InsertKey(s.keys, bits, x.idx[q]);
      }
      added += __popc(__ballot_sync(0xffffffffu, fresh));
    }
    __syncwarp();
  }
  return added;
}

template <class T>
struct SymbolicArgs {
  CscView<T> x;
  CscView<T> b;
  const int64_t* need;  // per column required slots
  bool add_diag;
  int64_t* counts;
  unsigned char* global_space;  // fallback workspace (nullptr: shared memory)
};

template <class T>
__global__ void SymbolicKernel(SymbolicArgs<T> a, int slots, int64_t lo_need, int64_t hi_need) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int warps_per_block = blockDim.x >> 5;
  const size_t bytes = SpaceBytes<T>(slots, false);
  unsigned char* base = a.global_space != nullptr
                            ? a.global_space + (static_cast<size_t>(blockIdx.x) * warps_per_block + warp_in_block) * bytes
                            : smem + warp_in_block * bytes;
  const Space<T> s = CarveSpace<T>(base, slots, false);
  const int bits = Log2(slots);
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t col = warp; col < a.b.cols; col += warps) {
    const int64_t need = a.need[col];
    if (need <= lo_need || need > hi_need) continue;
    ClearTable(s.keys, slots, lane);
    __syncwarp();
    const int count = InsertColumnRows(a.x, a.b, col, a.add_diag, s, bits, lane);
    if (lane == 0) a.counts[col] = count;
    __syncwarp();
  }
}

template <class T>
struct NumericArgs {
  CscView<T> x_csc;
  CscView<T> x_csr;
  CscView<T> b;
  const int64_t* need;
  const int64_t* c_ptr;  // symbolic offsets (nullptr for kProjection)
  int epilogue;
  int32_t* c_idx;
  T* c_val;
  T* z_val;
  const T* row_scale;
  double* col_squares;
  double* proj_tt;
  double* proj_bt;
  int64_t* kept;
  int32_t* flag;
  unsigned char* global_space;
};

template <class T>
__global__ void NumericKernel(NumericArgs<T> a, int slots, int64_t lo_need, int64_t hi_need) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int warps_per_block = blockDim.x >> 5;
  const size_t bytes = SpaceBytes<T>(slots, true);
  unsigned char* base = a.global_space != nullptr
                            ? a.global_space + (static_cast<size_t>(blockIdx.x) * warps_per_block + warp_in_block) * bytes
                            : smem + warp_in_block * bytes;
  const Space<T> s = CarveSpace<T>(base, slots, true);
  const int bits = Log2(slots);
  const int bbits = bits - 1;
  const int half = slots / 2;
  const bool residual = a.epilogue == static_cast<int>(Epilogue::kResidual);
  const bool projection = a.epilogue == static_cast<int>(Epilogue::kProjection);
  const bool prune = a.epilogue == static_cast<int>(Epilogue::kPruneZeros) || residual;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t col = warp; col < a.b.cols; col += warps) {
    const int64_t need = a.need[col];
    if (need <= lo_need || need > hi_need) continue;
    ClearTable(s.keys, slots, lane);
    ClearTable(s.bkeys, half, lane);
    __syncwarp();
    // hash of B(:, col): k -> value
    const int64_t bs = a.b.ptr[col];
    const int64_t be = a.b.ptr[col + 1];
    for (int64_t p = bs + lane; p < be; p += kWarp) {
      const uint32_t h = ClaimSlot(s.bkeys, bbits, a.b.idx[p]);
      s.bvals[h] = a.b.val[p];
    }
    InsertColumnRows(a.x_csc, a.b, col, residual, s, bits, lane);
    __syncwarp();
    // compact and sort the row set
    int count = 0;
    for (int base_slot = 0; base_slot < slots; base_slot += kWarp) {
      const int32_t key = s.keys[base_slot + lane];
      const bool occupied = key != kEmpty;
      const unsigned mask = __ballot_sync(0xffffffffu, occupied);
      if (occupied) s.sorted[count + __popc(mask & LaneMaskBelow())] = key;
      count += __popc(mask);
    }
    int size = 1;
    while (size < count) size <<= 1;
    for (int i = count + lane; i < size; i += kWarp) s.sorted[i] = INT32_MAX;
    __syncwarp();
    for (int k = 2; k <= size; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = lane; i < size; i += kWarp) {
          const int ixj = i ^ j;
          if (ixj > i) {
            const int32_t u = s.sorted[i];
            const int32_t v = s.sorted[ixj];
            const bool ascending = (i & k) == 0;
            if ((u > v) == ascending) {
              s.sorted[i] = v;
              s.sorted[ixj] = u;
            }
          }
        }
        __syncwarp();
      }
    }
    // numeric values
    const int64_t out_base = projection ? 0 : a.c_ptr[col];
    int kept = 0;
    for (int base_pos = 0; base_pos < count; base_pos += kWarp) {
      const int pos = base_pos + lane;
      const bool active = pos < count;
      int32_t row = 0;
      double acc = 0.0;
      bool has = false;
      if (active) {
        row = s.sorted[pos];
        const int64_t rs = a.x_csr.ptr[row];
        const int64_t re = a.x_csr.ptr[row + 1];
        for (int64_t q = rs; q < re; ++q) {
          T bv;
          if (Lookup(s.bkeys, s.bvals, bbits, a.x_csr.idx[q], bv)) {
            const double prod = Mul(static_cast<double>(a.x_csr.val[q]), static_cast<double>(bv));
            acc = has ? Add(acc, prod) : prod;
            has = true;
          }
        }
      }
      if (projection) {
        if (active) {
          const T az = static_cast<T>(acc);
          const T t = static_cast<T>(Mul(static_cast<double>(a.row_scale[row]), static_cast<double>(az)));
          const double td = static_cast<double>(t);
          s.stage0[pos] = Mul(td, td);
          T zv;
          const bool in_b = Lookup(s.bkeys, s.bvals, bbits, row, zv);
          s.present[pos] = in_b ? 1 : 0;
          s.stage1[pos] = in_b ? Mul(static_cast<double>(zv), td) : 0.0;
        }
        continue;
      }
      double v = acc;
      if (residual) {
        v = has ? -acc : 0.0;
        if (static_cast<int64_t>(row) == col) v = has ? Add(v, 1.0) : 1.0;
      }
      const T stored = static_cast<T>(v);
      const bool keep = active && !(prune && fabs(static_cast<double>(stored)) <= 0.0);
      const unsigned mask = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int slot = kept + __popc(mask & LaneMaskBelow());
        a.c_idx[out_base + slot] = row;
        a.c_val[out_base + slot] = stored;
        if (a.z_val != nullptr) {
          a.z_val[out_base + slot] =
              static_cast<T>(Mul(static_cast<double>(a.row_scale[row]), static_cast<double>(stored)));
        }
        const double sd = static_cast<double>(stored);
        s.stage0[slot] = Mul(sd, sd);
      }
      kept += __popc(mask);
    }
    __syncwarp();
    if (lane == 0) {
      if (projection) {
        double tt = 0.0;
        double bt = 0.0;
        for (int i = 0; i < count; ++i) {
          tt = Add(tt, s.stage0[i]);
          if (s.present[i]) bt = Add(bt, s.stage1[i]);
        }
        a.proj_tt[col] = tt;
        a.proj_bt[col] = bt;
      } else {
        if (a.col_squares != nullptr) {
          double sq = 0.0;
          for (int i = 0; i < kept; ++i) sq = Add(sq, s.stage0[i]);
          a.col_squares[col] = sq;
        }
        a.kept[col] = kept;
        if (kept != count) atomicOr(a.flag, 1);
      }
    }
    __syncwarp();
  }
}

template <class T>
struct MaskedArgs {
  CscView<T> x_csr;
  CscView<T> b;
  CscView<T> mask;
  const int64_t* need;
  double* out;
  unsigned char* global_space;
};

template <class T>
__global__ void MaskedKernel(MaskedArgs<T> a, int slots, int64_t lo_need, int64_t hi_need) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const int warp_in_block = threadIdx.x >> 5;
  const int warps_per_block = blockDim.x >> 5;
  const size_t bytes = SpaceBytes<T>(slots, true);
  unsigned char* base = a.global_space != nullptr
                            ? a.global_space + (static_cast<size_t>(blockIdx.x) * warps_per_block + warp_in_block) * bytes
                            : smem + warp_in_block * bytes;
  const Space<T> s = CarveSpace<T>(base, slots, true);
  const int bbits = Log2(slots) - 1;
  const int half = slots / 2;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t col = warp; col < a.b.cols; col += warps) {
    const int64_t need = a.need[col];
    if (need <= lo_need || need > hi_need) continue;
    ClearTable(s.bkeys, half, lane);
    __syncwarp();
    for (int64_t p = a.b.ptr[col] + lane; p < a.b.ptr[col + 1]; p += kWarp) {
      const uint32_t h = ClaimSlot(s.bkeys, bbits, a.b.idx[p]);
      s.bvals[h] = a.b.val[p];
    }
    __syncwarp();
    for (int64_t p = a.mask.ptr[col] + lane; p < a.mask.ptr[col + 1]; p += kWarp) {
      const int32_t row = a.mask.idx[p];
      double acc = 0.0;
      bool has = false;
      for (int64_t q = a.x_csr.ptr[row]; q < a.x_csr.ptr[row + 1]; ++q) {
        T bv;
        if (Lookup(s.bkeys, s.bvals, bbits, a.x_csr.idx[q], bv)) {
          const double prod = Mul(static_cast<double>(a.x_csr.val[q]), static_cast<double>(bv));
          acc = has ? Add(acc, prod) : prod;
          has = true;
        }
      }
      a.out[p] = has ? acc : 0.0;
    }
    __syncwarp();
  }
}

// One atomicMax per warp instead of one per thread.
__device__ __forceinline__ void WarpAtomicMax(unsigned long long* target, unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, v, o);
    v = other > v ? other : v;
  }
  if ((threadIdx.x & 31) == 0 && v != 0ull) atomicMax(target, v);
}

// upper bound on distinct rows and the B column length, plus the maxima.
template <class T>
__global__ void NeedKernel(CscView<T> x, CscView<T> b, bool add_diag, int64_t* __restrict__ ub,
                           unsigned long long* __restrict__ maxima) {
  unsigned long long local_ub = 0;
  unsigned long long local_nb = 0;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < b.cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t u = add_diag ? 1 : 0;
    for (int64_t p = b.ptr[j]; p < b.ptr[j + 1]; ++p) {
      const int32_t k = b.idx[p];
      u += x.ptr[k + 1] - x.ptr[k];
    }
    ub[j] = u;
    local_ub = max(local_ub, static_cast<unsigned long long>(u));
    local_nb = max(local_nb, static_cast<unsigned long long>(b.ptr[j + 1] - b.ptr[j]));
  }
  WarpAtomicMax(&maxima[0], local_ub);
  WarpAtomicMax(&maxima[1], local_nb);
}

// symbolic need = 2 * ub; numeric need = max(2 * count, 4 * nb)
__global__ void SymbolicNeedKernel(const int64_t* __restrict__ ub, int64_t cols, int64_t* __restrict__ need) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    need[j] = 2 * ub[j];
  }
}

__global__ void NumericNeedKernel(const int64_t* __restrict__ counts, const int64_t* __restrict__ bptr, int64_t cols,
                                  int64_t* __restrict__ need, unsigned long long* __restrict__ maxima) {
  unsigned long long local = 0;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t c = counts[j];
    const int64_t nb = bptr[j + 1] - bptr[j];
    int64_t v = 2 * c > 4 * nb ? 2 * c : 4 * nb;
    if (v < 2) v = 2;
    need[j] = v;
    local = max(local, static_cast<unsigned long long>(v));
  }
  WarpAtomicMax(&maxima[2], local);
}

__global__ void MaskedNeedKernel(const int64_t* __restrict__ bptr, int64_t cols, int64_t* __restrict__ need) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t v = 4 * (bptr[j + 1] - bptr[j]);
    need[j] = v < 2 ? 2 : v;
  }
}

template <class T>
__global__ void SqueezeKernel(int64_t cols, const int64_t* __restrict__ old_ptr, const int64_t* __restrict__ new_ptr,
                              const int32_t* __restrict__ old_idx, const T* __restrict__ old_val,
                              const T* __restrict__ old_z, int32_t* __restrict__ new_idx, T* __restrict__ new_val,
                              T* __restrict__ new_z) {
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < cols;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t src = old_ptr[j];
    const int64_t dst = new_ptr[j];
    const int64_t len = new_ptr[j + 1] - dst;
    for (int64_t i = 0; i < len; ++i) {
      new_idx[dst + i] = old_idx[src + i];
      new_val[dst + i] = old_val[src + i];
      if (new_z != nullptr) new_z[dst + i] = old_z[src + i];
    }
  }
}

struct Bin {
  int slots;
  int warps;
  int64_t lo;
  int64_t hi;
};

constexpr Bin kBins[] = {
    {256, 8, -1, 256},
    {1024, 4, 256, 1024},
    {4096, 1, 1024, 4096},
};
constexpr int64_t kLargestBin = 4096;

int NextPow2(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return static_cast<int>(p);
}

template <class Kernel, class Args>
void LaunchBins(Ctx& ctx, Kernel kernel, Args args, int64_t cols, int64_t max_need, bool numeric, size_t tsize,
                DevBuf<unsigned char>& fallback) {
  for (const Bin& bin : kBins) {
    if (max_need <= bin.lo) break;
    const size_t per_warp = numeric ? (tsize == 8 ? SpaceBytes<double>(bin.slots, true) : SpaceBytes<float>(bin.slots, true))
                                    : SpaceBytes<double>(bin.slots, false);
    const size_t smem = per_warp * bin.warps;
    SPAI_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    const int threads = bin.warps * kWarp;
    const int grid = GridFor(cols * kWarp, threads);
    args.global_space = nullptr;
    kernel<<<grid, threads, smem, ctx.stream>>>(args, bin.slots, bin.lo, bin.hi);
    SPAI_LAUNCH_CHECK();
  }
  if (max_need > kLargestBin) {
    const int slots = NextPow2(max_need);
    const size_t per_warp = numeric ? (tsize == 8 ? SpaceBytes<double>(slots, true) : SpaceBytes<float>(slots, true))
                                    : SpaceBytes<double>(slots, false);
    const int blocks = ctx.sm_count * 2;
    fallback.Reserve(per_warp * blocks, ctx.stream);
    args.global_space = fallback.data();
    kernel<<<blocks, kWarp, 0, ctx.stream>>>(args, slots, kLargestBin, INT64_MAX);
    SPAI_LAUNCH_CHECK();
  }
}

template <class T>
double MatrixBytes(int64_t nnz, int64_t major) {
  return static_cast<double>(nnz) * static_cast<double>(sizeof(T) + sizeof(int32_t)) +
         static_cast<double>(major + 1) * static_cast<double>(sizeof(int64_t));
}

}  // namespace

template <class T>
void Spgemm(Ctx& ctx, const DevCsc<T>& x_csc, const DevCsc<T>& x_csr, const DevCsc<T>& b, DevCsc<T>& c,
            Epilogue epilogue, SpgemmExtras extras, DevCsc<T>* c_z) {
  const int64_t cols = b.cols;
  const bool residual = epilogue == Epilogue::kResidual;
  const bool projection = epilogue == Epilogue::kProjection;
  DevBuf<int64_t> ub;
  DevBuf<int64_t> need;
  DevBuf<int64_t> counts;
  DevBuf<unsigned long long> maxima;
  DevBuf<unsigned char> fallback;
  ub.Reserve(static_cast<size_t>(cols), ctx.stream);
  need.Reserve(static_cast<size_t>(cols), ctx.stream);
  counts.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
  maxima.Reserve(4, ctx.stream);
  SPAI_CUDA(cudaMemsetAsync(maxima.data(), 0, 4 * sizeof(unsigned long long), ctx.stream));

  NeedKernel<T><<<GridFor(cols, 128), 128, 0, ctx.stream>>>(View(x_csc), View(b), residual, ub.data(), maxima.data());
  SPAI_LAUNCH_CHECK();
  SymbolicNeedKernel<<<GridFor(cols, 256), 256, 0, ctx.stream>>>(ub.data(), cols, need.data());
  SPAI_LAUNCH_CHECK();
  unsigned long long host_max[4];
  SPAI_CUDA(cudaMemcpyAsync(host_max, maxima.data(), sizeof(host_max), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();
  const int64_t max_sym_need = 2 * static_cast<int64_t>(host_max[0]);

  SymbolicArgs<T> sargs{View(x_csc), View(b), need.data(), residual, counts.data(), nullptr};
  {
    prof::Scope scope(ctx.stream, "spgemm_symbolic", 0.0);
    LaunchBins(ctx, SymbolicKernel<T>, sargs, cols, max_sym_need, false, sizeof(T), fallback);
  }

  NumericNeedKernel<<<GridFor(cols, 256), 256, 0, ctx.stream>>>(counts.data(), b.ptr.data(), cols, need.data(),
                                                                maxima.data());
  SPAI_LAUNCH_CHECK();

  DevCsc<T> result;
  DevBuf<T> zbuf;
  DevBuf<int64_t> kept;
  NumericArgs<T> nargs{};
  nargs.x_csc = View(x_csc);
  nargs.x_csr = View(x_csr);
  nargs.b = View(b);
  nargs.need = need.data();
  nargs.epilogue = static_cast<int>(epilogue);
  nargs.row_scale = static_cast<const T*>(extras.row_scale);
  nargs.col_squares = extras.col_squares;
  nargs.proj_tt = extras.proj_tt;
  nargs.proj_bt = extras.proj_bt;
  nargs.flag = ctx.flags.data();
  SPAI_CUDA(cudaMemsetAsync(ctx.flags.data(), 0, sizeof(int32_t), ctx.stream));
  int64_t nnz = 0;
  if (!projection) {
    result.Shape(x_csc.rows, cols, ctx.stream);
    nnz = ScanCounts(ctx, counts.data(), cols, result.ptr.data());
    result.ReserveNnz(nnz, ctx.stream);
    kept.Reserve(static_cast<size_t>(cols + 1), ctx.stream);
    nargs.c_ptr = result.ptr.data();
    nargs.c_idx = result.idx.data();
    nargs.c_val = result.val.data();
    nargs.kept = kept.data();
    if (extras.z_val != nullptr || c_z != nullptr) {
      zbuf.Reserve(static_cast<size_t>(nnz > 0 ? nnz : 1), ctx.stream);
      nargs.z_val = zbuf.data();
    }
  }
  SPAI_CUDA(cudaMemcpyAsync(host_max, maxima.data(), sizeof(host_max), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();
  const int64_t max_num_need = static_cast<int64_t>(host_max[2]);
  {
    // algorithmic bytes: |X| + |B| + |C| (C written; the projection writes two per-column sums instead)
    double bytes = MatrixBytes<T>(x_csr.nnz, x_csr.cols) + MatrixBytes<T>(b.nnz, b.cols);
    if (projection) {
      bytes += static_cast<double>(cols) * (sizeof(T) + 2 * sizeof(double));
    } else {
      bytes += MatrixBytes<T>(nnz, cols);
      if (nargs.z_val != nullptr) bytes += static_cast<double>(nnz) * sizeof(T);
    }
    prof::Scope scope(ctx.stream, "spgemm_numeric", bytes);
    LaunchBins(ctx, NumericKernel<T>, nargs, cols, max_num_need, true, sizeof(T), fallback);
  }
  if (projection) {
    return;
  }
  int32_t squeezed = 0;
  if (epilogue != Epilogue::kPlain) {
    SPAI_CUDA(cudaMemcpyAsync(ctx.host_flags, ctx.flags.data(), sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.Sync();
    squeezed = ctx.host_flags[0];
  }
  if (squeezed) {
    DevCsc<T> packed;
    packed.Shape(result.rows, cols, ctx.stream);
    const int64_t packed_nnz = ScanCounts(ctx, kept.data(), cols, packed.ptr.data());
    packed.ReserveNnz(packed_nnz, ctx.stream);
    DevBuf<T> packed_z;
    if (nargs.z_val != nullptr) packed_z.Reserve(static_cast<size_t>(packed_nnz > 0 ? packed_nnz : 1), ctx.stream);
    SqueezeKernel<T><<<GridFor(cols, 128), 128, 0, ctx.stream>>>(
        cols, result.ptr.data(), packed.ptr.data(), result.idx.data(), result.val.data(), zbuf.data(),
        packed.idx.data(), packed.val.data(), nargs.z_val != nullptr ? packed_z.data() : nullptr);
    SPAI_LAUNCH_CHECK();
    result.Swap(packed);
    zbuf.Swap(packed_z);
  }
  if (c_z != nullptr) {
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
}

template <class T>
void SpgemmMasked(Ctx& ctx, const DevCsc<T>& x_csr, const DevCsc<T>& b, const DevCsc<T>& mask, double* out) {
  const int64_t cols = b.cols;
  DevBuf<int64_t> need;
  DevBuf<unsigned char> fallback;
  need.Reserve(static_cast<size_t>(cols), ctx.stream);
  MaskedNeedKernel<<<GridFor(cols, 256), 256, 0, ctx.stream>>>(b.ptr.data(), cols, need.data());
  SPAI_LAUNCH_CHECK();
  // the largest B column decides whether the global workspace is needed
  DevBuf<unsigned long long> maxima;
  maxima.Reserve(4, ctx.stream);
  SPAI_CUDA(cudaMemsetAsync(maxima.data(), 0, 4 * sizeof(unsigned long long), ctx.stream));
  DevBuf<int64_t> ub;
  ub.Reserve(static_cast<size_t>(cols), ctx.stream);
  NeedKernel<T><<<GridFor(cols, 128), 128, 0, ctx.stream>>>(View(x_csr), View(b), false, ub.data(), maxima.data());
  SPAI_LAUNCH_CHECK();
  unsigned long long host_max[4];
  SPAI_CUDA(cudaMemcpyAsync(host_max, maxima.data(), sizeof(host_max), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();
  const int64_t max_need = std::max<int64_t>(2, 4 * static_cast<int64_t>(host_max[1]));
  MaskedArgs<T> args{View(x_csr), View(b), View(mask), need.data(), out, nullptr};
  LaunchBins(ctx, MaskedKernel<T>, args, cols, max_need, true, sizeof(T), fallback);
}

template void Spgemm<double>(Ctx&, const DevCsc<double>&, const DevCsc<double>&, const DevCsc<double>&,
                             DevCsc<double>&, Epilogue, SpgemmExtras, DevCsc<double>*);
template void Spgemm<float>(Ctx&, const DevCsc<float>&, const DevCsc<float>&, const DevCsc<float>&, DevCsc<float>&,
                            Epilogue, SpgemmExtras, DevCsc<float>*);
template void SpgemmMasked<double>(Ctx&, const DevCsc<double>&, const DevCsc<double>&, const DevCsc<double>&,
                                   double*);
template void SpgemmMasked<float>(Ctx&, const DevCsc<float>&, const DevCsc<float>&, const DevCsc<float>&, double*);

}  // namespace spai
