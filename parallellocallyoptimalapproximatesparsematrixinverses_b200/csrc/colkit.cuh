#pragma once
// Warp-per-column building blocks shared by the column kernels (spgemm.cu and
// the fused Global MR iteration, mr_fused.cu): a two-choice bucketed hash of
// one sparse column in shared memory, a two-level bitmap over a row window
// whose marked rows are read back in ascending order, and small helpers.

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "device.cuh"

namespace spai {

constexpr int32_t kEmpty = -1;  // empty hash slot

__device__ __forceinline__ unsigned LaneMaskBelow() {
  unsigned mask;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(mask));
  return mask;
}

__host__ __device__ inline int Log2(int v) {
  int b = 0;
  while ((1 << b) < v) ++b;
  return b;
}

__host__ __device__ inline size_t Round16(size_t v) { return (v + 15) & ~static_cast<size_t>(15); }

inline __device__ void ClearTable(int32_t* table, int size, int lane) {
  for (int i = lane; i < size; i += kWarp) table[i] = kEmpty;
}

inline __device__ void ClearWords(uint32_t* words, int size, int lane) {
  for (int i = lane; i < size; i += kWarp) words[i] = 0u;
}

__host__ __device__ inline int SummaryWords(int words) { return (words + kWarp * kWarp - 1) / (kWarp * kWarp) * kWarp; }

__device__ __forceinline__ void LoadFour(const float* p, float (&v)[4]) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  v[0] = q.x;
  v[1] = q.y;
  v[2] = q.z;
  v[3] = q.w;
}

__device__ __forceinline__ void LoadFour(const double* p, double (&v)[4]) {
  const double2 q0 = reinterpret_cast<const double2*>(p)[0];
  const double2 q1 = reinterpret_cast<const double2*>(p)[1];
  v[0] = q0.x;
  v[1] = q0.y;
  v[2] = q1.x;
  v[3] = q1.y;
}

// Two-choice bucketed hash of B(:,j): bucket = 2 slots (one 8-byte word of
// keys); a key lives in bucket h1 or h2 of its row, so a lookup is two
// fixed loads.  A key that finds both buckets full is placed by linear
// probing from the bucket after h2 (`displaced`, warp-uniform), and only
// then do lookups that miss both buckets continue probing.
__device__ __forceinline__ uint32_t Bucket1(int32_t key, int bits) {
  return (static_cast<uint32_t>(key) * 2654435761u) >> (32 - bits);
}

__device__ __forceinline__ uint32_t Bucket2(int32_t key, int bits, uint32_t h1) {
  const uint32_t h = (static_cast<uint32_t>(key) * 0x85EBCA6Bu + 0x9E3779B9u) >> (32 - bits);
  return h == h1 ? (h ^ 1u) & ((1u << bits) - 1u) : h;
}

// Returns false when the key had to be displaced.
template <class T>
__device__ __forceinline__ bool BucketInsert(int32_t* keys, T* vals, int bits, int32_t key, T v) {
  const uint32_t h1 = Bucket1(key, bits);
  const uint32_t h2 = Bucket2(key, bits, h1);
  const uint32_t slots[4] = {2 * h1, 2 * h1 + 1, 2 * h2, 2 * h2 + 1};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (atomicCAS(&keys[slots[i]], kEmpty, key) == kEmpty) {
      vals[slots[i]] = v;
      return true;
    }
  }
  const uint32_t mask = (2u << bits) - 1u;
  uint32_t s = (2 * h2 + 2) & mask;
  while (atomicCAS(&keys[s], kEmpty, key) != kEmpty) s = (s + 1u) & mask;
  vals[s] = v;
  return false;
}

template <class T>
__device__ __forceinline__ bool BucketFind(const int32_t* keys, const T* vals, int bits, bool displaced, int32_t key,
                                           T& out) {
  const uint32_t h1 = Bucket1(key, bits);
  const uint32_t h2 = Bucket2(key, bits, h1);
  const int2 a = reinterpret_cast<const int2*>(keys)[h1];
  const int2 b = reinterpret_cast<const int2*>(keys)[h2];
  int slot = b.y == key ? static_cast<int>(2 * h2 + 1) : -1;
  slot = b.x == key ? static_cast<int>(2 * h2) : slot;
  slot = a.y == key ? static_cast<int>(2 * h1 + 1) : slot;
  slot = a.x == key ? static_cast<int>(2 * h1) : slot;
  if (slot < 0 && displaced) {
    const uint32_t mask = (2u << bits) - 1u;
    uint32_t s = (2 * h2 + 2) & mask;
    while (true) {
      const int32_t k = keys[s];
      if (k == key) {
        slot = static_cast<int>(s);
        break;
      }
      if (k == kEmpty) break;
      s = (s + 1u) & mask;
    }
  }
  if (slot < 0) return false;
  out = vals[slot];
  return true;
}

// Marks `off` in the two-level bitmap.
__device__ __forceinline__ void MarkRow(uint32_t* bm, uint32_t* summary, int off) {
  const int w = off >> 5;
  const uint32_t old = atomicOr(&bm[w], 1u << (off & 31));
  if (old == 0u) atomicOr(&summary[w >> 5], 1u << (w & 31));
}

// Reads the marked rows back in ascending order, as 16-bit offsets from the
// window start (a window spans at most 65,536 rows), into rows[] unless null,
// clearing both levels; returns the warp-uniform count.
inline __device__ int DrainRows(uint32_t* bm, uint32_t* summary, int summary_words, uint16_t* rows, int lane) {
  int total = 0;
  for (int s0 = 0; s0 < summary_words; s0 += kWarp) {
    const int s = s0 + lane;
    const uint32_t sbits = summary[s];
    int local = 0;
    for (uint32_t t = sbits; t != 0u; t &= t - 1u) local += __popc(bm[(s << 5) + __ffs(t) - 1]);
    int inclusive = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, inclusive, o);
      if (lane >= o) inclusive += y;
    }
    int at = total + inclusive - local;
    for (uint32_t t = sbits; t != 0u; t &= t - 1u) {
      const int w = (s << 5) + __ffs(t) - 1;
      uint32_t bits = bm[w];
      bm[w] = 0u;
      if (rows != nullptr) {
        for (; bits != 0u; bits &= bits - 1u) rows[at++] = static_cast<uint16_t>((w << 5) + (__ffs(bits) - 1));
      }
    }
    summary[s] = 0u;
    total += __shfl_sync(0xffffffffu, inclusive, 31);
  }
  __syncwarp();
  return total;
}

}  // namespace spai
