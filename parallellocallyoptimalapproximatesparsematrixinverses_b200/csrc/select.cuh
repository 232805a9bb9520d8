#pragma once
// The drop step's per-column selection, shared by the symmetrize-and-drop
// kernel (update.cu) and the fused Global MR iteration (mr_fused.cu): a
// merged column of S = 0.5 (M + M^T) staged in a per-warp shared-memory slab,
// the relative threshold and the per-column top-k by (|v|, row).

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "colkit.cuh"
#include "device.cuh"

namespace spai {

// First position in keys[0, n) whose row is >= key (keys in shared memory).
__device__ __forceinline__ int LowerBoundShared(const int32_t* keys, int n, int32_t key) {
  int lo = 0;
  int hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (keys[mid] < key) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

constexpr int kDropCap = 256;        // longest merged column of the fused drop kernel
constexpr double kDblEps = 2.220446049250313080847e-16;

// Per-warp shared memory of the fused drop kernel: the merged column (keys,
// vals, keep), the matched prefix, and the row indices of both input columns.
struct DropSlab {
  double* vals;
  int32_t* keys;
  int* mx_prefix;
  unsigned char* keep;
  int32_t* yk;
  int32_t* xk;
};

__host__ __device__ constexpr size_t Round16Bytes(size_t v) { return (v + 15) & ~size_t(15); }

__host__ __device__ constexpr size_t DropSlabBytes() {
  return Round16Bytes(kDropCap * sizeof(double)) + Round16Bytes(kDropCap * sizeof(int32_t)) +
         Round16Bytes((kDropCap + 1) * sizeof(int)) + Round16Bytes(kDropCap) + 2 * Round16Bytes(kDropCap * 4);
}

inline __device__ DropSlab SlabFor(unsigned char* base) {
  DropSlab s;
  s.vals = reinterpret_cast<double*>(base);
  base += Round16Bytes(kDropCap * sizeof(double));
  s.keys = reinterpret_cast<int32_t*>(base);
  base += Round16Bytes(kDropCap * sizeof(int32_t));
  s.mx_prefix = reinterpret_cast<int*>(base);
  base += Round16Bytes((kDropCap + 1) * sizeof(int));
  s.keep = base;
  base += Round16Bytes(kDropCap);
  s.yk = reinterpret_cast<int32_t*>(base);
  base += Round16Bytes(kDropCap * 4);
  s.xk = reinterpret_cast<int32_t*>(base);
  return s;
}

// (|v| bits, position) ordering; the position breaks ties exactly as the row does.
__device__ __forceinline__ bool KeyGreater(unsigned long long a, uint32_t pa, unsigned long long b, uint32_t pb) {
  return a > b || (a == b && pa > pb);
}

// Ascending bitonic sort of 32*R (key, position) pairs held as element
// t*32 + lane in register t of each lane.
template <int R>
__device__ __forceinline__ void WarpBitonicSort(unsigned long long (&k)[R], uint32_t (&p)[R], int lane) {
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
            if (KeyGreater(k[t], p[t], k[u], p[u]) == up) {
              const unsigned long long kk = k[t];
              k[t] = k[u];
              k[u] = kk;
              const uint32_t pp = p[t];
              p[t] = p[u];
              p[u] = pp;
            }
          }
        }
      } else {
#pragma unroll
        for (int t = 0; t < R; ++t) {
          const unsigned long long ok = __shfl_xor_sync(0xffffffffu, k[t], stride);
          const uint32_t op = __shfl_xor_sync(0xffffffffu, p[t], stride);
          const bool up = ((t * kWarp + lane) & size) == 0;
          const bool lower = (lane & stride) == 0;
          const bool mine_greater = KeyGreater(k[t], p[t], ok, op);
          // the lower slot of an ascending pair keeps the smaller element
          if (mine_greater == (lower == up)) {
            k[t] = ok;
            p[t] = op;
          }
        }
      }
    }
  }
}

// Marks the `drop` smallest (|v|, row) kept off-diagonal entries of the
// column held in the slab as dropped; count <= 32 * R.
template <int R>
inline __device__ void DropSmallest(DropSlab& s, int count, int64_t col, int drop, int lane) {
  unsigned long long k[R];
  uint32_t p[R];
#pragma unroll
  for (int t = 0; t < R; ++t) {
    const int e = t * kWarp + lane;
    const bool candidate = e < count && s.keep[e] != 0 && static_cast<int64_t>(s.keys[e]) != col;
    k[t] = candidate ? static_cast<unsigned long long>(__double_as_longlong(fabs(s.vals[e]))) : ~0ull;
    p[t] = static_cast<uint32_t>(e);
  }
  WarpBitonicSort<R>(k, p, lane);
  __syncwarp();
#pragma unroll
  for (int t = 0; t < R; ++t) {
    if (t * kWarp + lane < drop) s.keep[p[t]] = 0;
  }
  __syncwarp();
}

// Keeps the keep_off largest (|v|, row) kept off-diagonal entries of the
// column in the slab and marks the other candidates dropped.  Exact
// prefilter: the keep_off-th largest of the 32 per-lane maxima bounds the
// cut from below, so only candidates at or above it (usually <= 32) are
// sorted; otherwise the full sort of DropSmallest decides.
template <int R>
inline __device__ void KeepLargest(DropSlab& s, int count, int64_t col, int candidates, int keep_off, int lane) {
  if (keep_off == 0) {
    for (int e = lane; e < count; e += kWarp) {
      if (s.keep[e] != 0 && static_cast<int64_t>(s.keys[e]) != col) s.keep[e] = 0;
    }
    __syncwarp();
    return;
  }
  unsigned long long k[R];
  uint32_t p[R];
  unsigned long long best = 0ull;
  uint32_t best_p = 0u;
#pragma unroll
  for (int t = 0; t < R; ++t) {
    const int e = t * kWarp + lane;
    const bool candidate = e < count && s.keep[e] != 0 && static_cast<int64_t>(s.keys[e]) != col;
    // candidates have |v| > 0, so 0 sorts every other slot below them
    k[t] = candidate ? static_cast<unsigned long long>(__double_as_longlong(fabs(s.vals[e]))) : 0ull;
    p[t] = static_cast<uint32_t>(e);
    if (KeyGreater(k[t], p[t], best, best_p)) {
      best = k[t];
      best_p = p[t];
    }
  }
  if (keep_off <= kWarp) {
    unsigned long long m[1] = {best};
    uint32_t mp[1] = {best_p};
    WarpBitonicSort<1>(m, mp, lane);
    const unsigned long long cut = __shfl_sync(0xffffffffu, m[0], kWarp - keep_off);
    const uint32_t cut_p = __shfl_sync(0xffffffffu, mp[0], kWarp - keep_off);
    int survivors = 0;
    bool mine[R];
#pragma unroll
    for (int t = 0; t < R; ++t) {
      mine[t] = k[t] != 0ull && !KeyGreater(cut, cut_p, k[t], p[t]);
      survivors += __popc(__ballot_sync(0xffffffffu, mine[t]));
    }
    if (survivors <= kWarp) {
      // gather the survivors into one register per lane, staged in the
      // (no longer needed) input-key area of the slab
      unsigned long long* stage_k = reinterpret_cast<unsigned long long*>(s.xk);
      uint32_t* stage_p = reinterpret_cast<uint32_t*>(s.xk + 2 * kWarp);
      int filled = 0;
#pragma unroll
      for (int t = 0; t < R; ++t) {
        const unsigned mask = __ballot_sync(0xffffffffu, mine[t]);
        if (mine[t]) {
          const int at = filled + __popc(mask & LaneMaskBelow());
          stage_k[at] = k[t];
          stage_p[at] = p[t];
        }
        filled += __popc(mask);
      }
      __syncwarp();
      unsigned long long gk[1] = {lane < filled ? stage_k[lane] : 0ull};
      // padding sorts below every survivor and is never marked
      uint32_t gpp[1] = {lane < filled ? stage_p[lane] : 0xFFFF0000u + static_cast<uint32_t>(lane)};
      __syncwarp();
      WarpBitonicSort<1>(gk, gpp, lane);
      // every candidate is dropped except the keep_off largest survivors
#pragma unroll
      for (int t = 0; t < R; ++t) {
        if (k[t] != 0ull) s.keep[p[t]] = 0;
      }
      __syncwarp();
      if (lane >= kWarp - keep_off && gpp[0] < 0xFFFF0000u) s.keep[gpp[0]] = 1;
      __syncwarp();
      return;
    }
  }
  DropSmallest<R>(s, count, col, candidates - keep_off, lane);
}

// The drop decision for one merged column held in the slab (count entries,
// rows ascending; the reference's dropping.cpp:122-135 plus the per-column
// top-k): the relative threshold eps * ||S(:, j)||_2 with the squares summed
// in row order by one lane, the diagonal always kept, exact zeros dropped,
// then at most topk entries (topk > 0) by the largest (|v|, row).  Leaves
// s.keep[i] set for the survivors and returns their number.
inline __device__ int DecideDrops(DropSlab& s, int count, int64_t j, int64_t topk, int lane) {
  double thr = 0.0;
  if (lane == 0) {
    double sq = 0.0;
    const double2* v2 = reinterpret_cast<const double2*>(s.vals);
    int i = 0;
    for (; i + 1 < count; i += 2) {
      const double2 v = v2[i >> 1];
      sq = Add(sq, Mul(v.x, v.x));
      sq = Add(sq, Mul(v.y, v.y));
    }
    if (i < count) sq = Add(sq, Mul(s.vals[i], s.vals[i]));
    thr = Mul(kDblEps, sqrt(sq));
  }
  thr = __shfl_sync(0xffffffffu, thr, 0);
  int kept = 0;
  bool has_diag = false;
  for (int base = 0; base < count; base += kWarp) {
    const int i = base + lane;
    bool keep = false;
    bool diag = false;
    if (i < count) {
      const double v = s.vals[i];
      diag = static_cast<int64_t>(s.keys[i]) == j;
      keep = v != 0.0 && (diag || fabs(v) >= thr);
      s.keep[i] = keep ? 1 : 0;
    }
    kept += __popc(__ballot_sync(0xffffffffu, keep));
    if (__any_sync(0xffffffffu, keep && diag)) has_diag = true;
  }
  __syncwarp();
  if (topk > 0 && kept > topk) {
    // drop the smallest (|v|, row) among the kept off-diagonal entries
    const int64_t candidates = kept - (has_diag ? 1 : 0);
    const int64_t keep_off = topk - (has_diag ? 1 : 0) > 0 ? topk - (has_diag ? 1 : 0) : 0;
    const int drop = static_cast<int>(candidates - keep_off);
    if (drop > 0) {
      const int c = static_cast<int>(candidates);
      const int ko = static_cast<int>(keep_off);
      if (count <= kWarp) {
        KeepLargest<1>(s, count, j, c, ko, lane);
      } else if (count <= 2 * kWarp) {
        KeepLargest<2>(s, count, j, c, ko, lane);
      } else if (count <= 4 * kWarp) {
        KeepLargest<4>(s, count, j, c, ko, lane);
      } else {
        KeepLargest<8>(s, count, j, c, ko, lane);
      }
      kept -= drop;
    }
  }
  return kept;
}

}  // namespace spai
