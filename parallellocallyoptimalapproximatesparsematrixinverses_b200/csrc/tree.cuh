#pragma once
// The canonical reduction tree of the library (the "device summation order"):
// values are summed in chunks of kTreeChunk = 4096, lane t of kTreeLanes = 256
// adding values t, t + 256, ... of its chunk in order, then a fixed butterfly
// over the 256 lane sums; chunk sums are reduced again by the same rule until
// one value is left.  The CPU oracle restates exactly this order, so every
// kernel that forms a tree level must use these helpers.

#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"

namespace spai {

constexpr int kTreeLanes = 256;
constexpr int64_t kTreeChunk = 4096;
constexpr int kTreeTerms = static_cast<int>(kTreeChunk / kTreeLanes);  // 16 terms per lane

// The lanes' partial sums of one chunk -> the chunk's sum: a butterfly over
// the kTreeLanes threads of the block (every thread returns the sum).  The
// block must have exactly kTreeLanes threads; `shared` holds kTreeLanes doubles.
__device__ __forceinline__ double TreeButterfly(double s, double* shared) {
  const int t = threadIdx.x;
  shared[t] = s;
  __syncthreads();
#pragma unroll
  for (int stride = kTreeLanes / 2; stride >= kWarp; stride >>= 1) {
    const double other = shared[t ^ stride];
    __syncthreads();
    s = Add(s, other);
    shared[t] = s;
    __syncthreads();
  }
#pragma unroll
  for (int stride = kWarp / 2; stride >= 1; stride >>= 1) {
    s = Add(s, __shfl_xor_sync(0xffffffffu, s, stride));
  }
  return s;
}

// One tree level over `count` <= kTreeChunk values already in global memory
// (written by other blocks of the running grid: read past L1), by the
// kTreeLanes threads of one block; every thread returns the sum.
__device__ __forceinline__ double TreeLevel(const double* values, int64_t count, double* shared) {
  const int t = threadIdx.x;
  double s = 0.0;
#pragma unroll
  for (int m = 0; m < kTreeTerms; ++m) {
    const int64_t i = t + static_cast<int64_t>(kTreeLanes) * m;
    if (i < count) s = Add(s, __ldcg(values + i));
  }
  return TreeButterfly(s, shared);
}

}  // namespace spai
