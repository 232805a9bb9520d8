// spai_pcg_device_noalloc: the PCG evaluator for callers that cannot let a
// library allocate.
//
// Who needs it: a simulation or solver loop that has handed the device's
// memory to its own pool (allocations from anyone else fail or evict its
// working set), or one that must not stall its other streams -- cudaFree
// synchronises the whole device, and a growing allocation can too.  Such a
// caller keeps A, M, b and x in its own device buffers and calls this entry
// point every step.
//
// How it allocates nothing: the four work vectors (r, z, p, A p), the
// first-level sums of the dot-product tree and the status word live in one
// fixed array in the library's device data (g_noalloc_scratch below,
// 16 MiB + 1.1 KiB), which the CUDA module carries.  In host code the array's
// name is only a host-side stand-in, so every call asks the runtime for the
// array's device address in the current context (cudaGetSymbolAddress, a
// table lookup once the module is loaded).  Asking on every call, instead of
// caching the address per device ordinal, keeps the address right after
// cudaDeviceReset or when the caller makes another context current.  The
// first call on a device can load the library's device code there and so
// must come before any stream capture on it.  Problems with more than
// kNoAllocMaxRows rows are rejected with an error.  The host side uses only
// stack memory and the caller's buffers; scalars come back through plain
// device-to-host copies into stack variables, so the call is
// host-synchronous: it waits for the stream about three times per iteration.
//
// Calls share the one scratch array per device: two calls that overlap on the
// same GPU (different streams, or different host threads) race and corrupt
// each other's vectors.  Serialise calls per device.  x must not overlap b,
// A or M (x is cleared before r = b is formed); such calls are rejected.
//
// The arithmetic is that of spai_pcg with FP64 M (pcg.cu, the reference's
// methods_cython/backward_error.pyx:69-144): per-row sequential SpMV, the
// fixed 4096-wide dot-product tree, the same recurrences and refresh rule, so
// both entry points return the same bits.

#include <cuda.h>  // driver types for the address-range query (no link-time dependency)
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "device.cuh"

namespace spai {
namespace {

constexpr int64_t kNoAllocMaxRows = 524288;  // 2^19 rows (an 80^3 grid fits)
constexpr int kTreeLanes = 256;
constexpr int64_t kTreeChunk = 4096;
constexpr int64_t kChunkSums = kNoAllocMaxRows / kTreeChunk;  // 128
// scratch layout, in doubles: r | z | p | ap | chunk sums | scalar | status
constexpr int64_t kOffR = 0;
constexpr int64_t kOffZ = kNoAllocMaxRows;
constexpr int64_t kOffP = 2 * kNoAllocMaxRows;
constexpr int64_t kOffAp = 3 * kNoAllocMaxRows;
constexpr int64_t kOffChunks = 4 * kNoAllocMaxRows;
constexpr int64_t kOffScalar = kOffChunks + kChunkSums;
constexpr int64_t kOffStatus = kOffScalar + 8;
constexpr int64_t kScratchDoubles = kOffStatus + 8;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
int g_sm_count_of_device[kMaxDevices] = {};  // 0 until the device's first call

// Status bits written by the input check.
constexpr unsigned long long kBadA = 1ull;
constexpr unsigned long long kBadM = 2ull;

__global__ void CheckCsrKernel(int64_t n, int64_t nnz, const int64_t* __restrict__ offsets,
                               const int32_t* __restrict__ indices, unsigned long long bad_bit,
                               unsigned long long* __restrict__ status) {
  for (int64_t row = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; row < n;
       row += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t o0 = offsets[row];
    const int64_t o1 = offsets[row + 1];
    bool bad = (row == 0 && o0 != 0) || (row == n - 1 && o1 != nnz) || o0 < 0 || o1 < o0 || o1 > nnz;
    if (!bad) {
      for (int64_t k = o0; k < o1; ++k) {
        const int32_t c = indices[k];
        if (c < 0 || static_cast<int64_t>(c) >= n) {
          bad = true;
          break;
        }
      }
    }
    if (bad) atomicOr(status, bad_bit);
  }
}

// y = A x, one thread per row, entries in storage order.
__global__ void NoAllocSpmvKernel(int64_t n, const int64_t* __restrict__ offsets, const int32_t* __restrict__ indices,
                                  const double* __restrict__ values, const double* __restrict__ x,
                                  double* __restrict__ y) {
  for (int64_t row = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; row < n;
       row += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int64_t k = offsets[row]; k < offsets[row + 1]; ++k) s = Add(s, Mul(values[k], x[indices[k]]));
    y[row] = s;
  }
}

__global__ void NoAllocStepKernel(int64_t n, double alpha, const double* __restrict__ p,
                                  const double* __restrict__ ap, double* __restrict__ x, double* __restrict__ r) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    x[i] = Add(x[i], Mul(alpha, p[i]));
    r[i] = __dsub_rn(r[i], Mul(alpha, ap[i]));
  }
}

__global__ void NoAllocResidualKernel(int64_t n, const double* __restrict__ b, const double* __restrict__ ax,
                                      double* __restrict__ r) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    r[i] = __dsub_rn(b[i], ax[i]);
  }
}

__global__ void NoAllocDirectionKernel(int64_t n, double beta, const double* __restrict__ z, double* __restrict__ p) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    p[i] = Add(z[i], Mul(beta, p[i]));
  }
}

// One 4096-value chunk of the dot-product tree: lane t sums terms t, t+256,
// ... in order, then a fixed butterfly over the 256 lane sums.  y == nullptr
// sums x itself (the upper tree level).
__global__ void NoAllocTreeKernel(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                                  double* __restrict__ out) {
  __shared__ double shared[kTreeLanes];
  const int t = threadIdx.x;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTreeChunk + t;
  double s = 0.0;
  if (y != nullptr) {
#pragma unroll
    for (int m = 0; m < static_cast<int>(kTreeChunk / kTreeLanes); ++m) {
      const int64_t i = base + static_cast<int64_t>(kTreeLanes) * m;
      if (i < n) s = Add(s, Mul(x[i], y[i]));
    }
  } else {
#pragma unroll
    for (int m = 0; m < static_cast<int>(kTreeChunk / kTreeLanes); ++m) {
      const int64_t i = base + static_cast<int64_t>(kTreeLanes) * m;
      if (i < n) s = Add(s, x[i]);
    }
  }
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
  for (int stride = kWarp / 2; stride >= 1; stride >>= 1) s = Add(s, __shfl_xor_sync(0xffffffffu, s, stride));
  if (t == 0) out[blockIdx.x] = s;
}

void SetError(char* error, int64_t capacity, const char* format, ...) {
  if (error == nullptr || capacity <= 0) return;
  va_list args;
  va_start(args, format);
  std::vsnprintf(error, static_cast<size_t>(capacity), format, args);
  va_end(args);
}

// Everything one call needs; every failure is recorded in `error` and turns
// the remaining steps into no-ops.
struct NoAllocRun {
  cudaStream_t stream;
  int64_t n;
  int grid;
  double* scratch;
  char* error;
  int64_t capacity;
  bool failed = false;

  bool Ok(cudaError_t err, const char* what) {
    if (failed) return false;
    if (err != cudaSuccess) {
      SetError(error, capacity, "CUDA error: %s (%s)", cudaGetErrorString(err), what);
      failed = true;
      return false;
    }
    return true;
  }
  bool Launched(const char* what) {
    CountLaunch();
    return Ok(cudaGetLastError(), what);
  }

  void Spmv(const int64_t* offsets, const int32_t* indices, const double* values, const double* x, double* y) {
    if (failed) return;
    NoAllocSpmvKernel<<<grid, 128, 0, stream>>>(n, offsets, indices, values, x, y);
    Launched("spmv");
  }

  double Dot(const double* x, const double* y) {
    double out = 0.0;
    if (failed) return out;
    const int64_t chunks = CeilDiv(n, kTreeChunk);
    double* scalar = scratch + kOffScalar;
    if (chunks == 1) {
      NoAllocTreeKernel<<<1, kTreeLanes, 0, stream>>>(x, y, n, scalar);
      Launched("dot");
    } else {
      double* sums = scratch + kOffChunks;
      NoAllocTreeKernel<<<static_cast<unsigned>(chunks), kTreeLanes, 0, stream>>>(x, y, n, sums);
      if (!Launched("dot")) return out;
      NoAllocTreeKernel<<<1, kTreeLanes, 0, stream>>>(sums, nullptr, chunks, scalar);
      Launched("dot");
    }
    if (!Ok(cudaMemcpyAsync(&out, scalar, sizeof(double), cudaMemcpyDeviceToHost, stream), "dot readback")) return out;
    Ok(cudaStreamSynchronize(stream), "dot readback");
    return out;
  }
};

// cuMemGetAddressRange, fetched through the runtime once per process (null
// when unavailable); resolved under std::call_once before any reader sees it.
using AddressRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
AddressRangeFn g_address_range = nullptr;
std::once_flag g_address_range_once;

AddressRangeFn AddressRange() {
  std::call_once(g_address_range_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &fn, 12000, cudaEnableDefault, &found) ==
            cudaSuccess &&
        found == cudaDriverEntryPointSuccess) {
      g_address_range = reinterpret_cast<AddressRangeFn>(fn);
    } else {
      cudaGetLastError();
    }
  });
  return g_address_range;
}

// True when [ptr, ptr + bytes) is device (or managed) memory usable on
// `device` and lies inside one allocation; otherwise fills `error`.
bool CheckDeviceExtent(const void* ptr, size_t bytes, int device, const char* name, char* error, int64_t capacity) {
  if (bytes == 0) return true;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
    cudaGetLastError();
    SetError(error, capacity, "%s is not a pointer CUDA knows", name);
    return false;
  }
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) {
    SetError(error, capacity, "%s must point to device memory", name);
    return false;
  }
  if (attr.type == cudaMemoryTypeDevice && attr.device != device) {
    SetError(error, capacity, "%s lives on device %d but device %d is current", name, attr.device, device);
    return false;
  }
  const AddressRangeFn address_range = AddressRange();
  if (address_range != nullptr) {
    CUdeviceptr base = 0;
    size_t size = 0;
    if (address_range(&base, &size, reinterpret_cast<CUdeviceptr>(ptr)) != CUDA_SUCCESS) {
      SetError(error, capacity, "the allocation holding %s is unknown to the driver", name);
      return false;
    }
    if (reinterpret_cast<uintptr_t>(ptr) + bytes > static_cast<uintptr_t>(base) + size) {
      SetError(error, capacity, "%s is shorter than the %zu bytes it must hold", name, bytes);
      return false;
    }
  }
  return true;
}

// The scratch array's device address in the current context, looked up on
// every call (never cached: a cached address goes stale when the context is
// reset or replaced), and the device's SM count, read on its first call.
double* ScratchOfDevice(int device, int* sm_count, char* error, int64_t capacity) {
  void* address = nullptr;
  cudaError_t err = cudaGetSymbolAddress(&address, g_noalloc_scratch);
  if (err != cudaSuccess || address == nullptr) {
    cudaGetLastError();
    SetError(error, capacity, "CUDA error: %s (cudaGetSymbolAddress of the no-alloc scratch)",
             cudaGetErrorString(err));
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_sm_count_of_device[device] == 0) {
    int sms = 0;
    err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err != cudaSuccess || sms <= 0) {
      cudaGetLastError();
      SetError(error, capacity, "CUDA error: %s (multiprocessor count)", cudaGetErrorString(err));
      return nullptr;
    }
    g_sm_count_of_device[device] = sms;
  }
  *sm_count = g_sm_count_of_device[device];
  return static_cast<double*>(address);
}

// True when the byte ranges [a, a + a_bytes) and [b, b + b_bytes) share a byte.
bool Overlaps(const void* a, size_t a_bytes, const void* b, size_t b_bytes) {
  if (a == nullptr || b == nullptr || a_bytes == 0 || b_bytes == 0) return false;
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(a);
  const uintptr_t b0 = reinterpret_cast<uintptr_t>(b);
  return a0 < b0 + b_bytes && b0 < a0 + a_bytes;
}

int GridOf(int64_t items, int threads, int sm_count) {
  const int64_t need = CeilDiv(items, threads);
  const int64_t cap = static_cast<int64_t>(sm_count) * 8;
  const int64_t grid = need < cap ? need : cap;
  return static_cast<int>(grid > 0 ? grid : 1);
}

}  // namespace
}  // namespace spai

extern "C" int64_t spai_pcg_device_noalloc(int64_t n, int64_t a_nnz, const double* a_values, const int32_t* a_indices,
                                           const int64_t* a_offsets, int64_t m_nnz, const double* m_values,
                                           const int32_t* m_indices, const int64_t* m_offsets, const double* b,
                                           double* x, int64_t max_iterations, double tolerance,
                                           int64_t refresh_period, void* stream, double* history, int64_t* status,
                                           char* error, int64_t error_capacity) {
  using namespace spai;
  if (n <= 0 || max_iterations <= 0) {
    SetError(error, error_capacity, "n and max_iterations must be positive");
    return -1;
  }
  if (n > kNoAllocMaxRows) {
    SetError(error, error_capacity,
             "n = %lld exceeds the no-alloc maximum of %lld rows (use spai_pcg or spai_session_pcg)",
             static_cast<long long>(n), static_cast<long long>(kNoAllocMaxRows));
    return -1;
  }
  if (a_nnz < 0 || m_nnz < 0) {
    SetError(error, error_capacity, "a_nnz and m_nnz must be non-negative");
    return -1;
  }
  if (!(tolerance >= 0.0) || refresh_period < 0) {
    SetError(error, error_capacity, "tolerance must be non-negative and refresh_period non-negative");
    return -1;
  }
  if (a_offsets == nullptr || m_offsets == nullptr || b == nullptr || x == nullptr || history == nullptr ||
      (a_nnz > 0 && (a_values == nullptr || a_indices == nullptr)) ||
      (m_nnz > 0 && (m_values == nullptr || m_indices == nullptr))) {
    SetError(error, error_capacity, "a required pointer is NULL");
    return -1;
  }
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) {
    SetError(error, error_capacity, "CUDA error: %s (cudaGetDevice)", cudaGetErrorString(err));
    return -1;
  }
  if (device < 0 || device >= kMaxDevices) {
    SetError(error, error_capacity, "device ordinal %d is beyond the no-alloc table", device);
    return -1;
  }
  int sm_count = 0;
  double* scratch = ScratchOfDevice(device, &sm_count, error, error_capacity);
  if (scratch == nullptr) return -1;

  // every device buffer must be on this device and long enough for what the kernels read or write
  const size_t vec = sizeof(double) * static_cast<size_t>(n);
  const size_t offs = sizeof(int64_t) * static_cast<size_t>(n + 1);
  if (!CheckDeviceExtent(a_offsets, offs, device, "a_offsets", error, error_capacity) ||
      !CheckDeviceExtent(a_indices, sizeof(int32_t) * static_cast<size_t>(a_nnz), device, "a_indices", error,
                         error_capacity) ||
      !CheckDeviceExtent(a_values, sizeof(double) * static_cast<size_t>(a_nnz), device, "a_values", error,
                         error_capacity) ||
      !CheckDeviceExtent(m_offsets, offs, device, "m_offsets", error, error_capacity) ||
      !CheckDeviceExtent(m_indices, sizeof(int32_t) * static_cast<size_t>(m_nnz), device, "m_indices", error,
                         error_capacity) ||
      !CheckDeviceExtent(m_values, sizeof(double) * static_cast<size_t>(m_nnz), device, "m_values", error,
                         error_capacity) ||
      !CheckDeviceExtent(b, vec, device, "b", error, error_capacity) ||
      !CheckDeviceExtent(x, vec, device, "x", error, error_capacity)) {
    return -1;
  }
  // x is cleared before r = b is formed and written every iteration: it must alias no input
  const struct {
    const void* ptr;
    size_t bytes;
    const char* name;
  } inputs[] = {{b, vec, "b"},
                {a_offsets, offs, "a_offsets"},
                {a_indices, sizeof(int32_t) * static_cast<size_t>(a_nnz), "a_indices"},
                {a_values, sizeof(double) * static_cast<size_t>(a_nnz), "a_values"},
                {m_offsets, offs, "m_offsets"},
                {m_indices, sizeof(int32_t) * static_cast<size_t>(m_nnz), "m_indices"},
                {m_values, sizeof(double) * static_cast<size_t>(m_nnz), "m_values"}};
  for (const auto& in : inputs) {
    if (Overlaps(x, vec, in.ptr, in.bytes)) {
      SetError(error, error_capacity, "x overlaps %s: x must not alias any input", in.name);
      return -1;
    }
  }

  // SpMV launches use 128 threads per block, the vector updates 256
  NoAllocRun run{static_cast<cudaStream_t>(stream), n, GridOf(n, 128, sm_count), scratch, error, error_capacity};
  double* r = scratch + kOffR;
  double* z = scratch + kOffZ;
  double* p = scratch + kOffP;
  double* ap = scratch + kOffAp;
  auto* check = reinterpret_cast<unsigned long long*>(scratch + kOffStatus);

  // inputs: offsets from 0 to nnz, non-decreasing, column indices inside [0, n)
  run.Ok(cudaMemsetAsync(check, 0, sizeof(unsigned long long), run.stream), "clear status");
  if (!run.failed) {
    CheckCsrKernel<<<GridOf(n, 128, sm_count), 128, 0, run.stream>>>(n, a_nnz, a_offsets, a_indices, kBadA, check);
    run.Launched("check A");
  }
  if (!run.failed) {
    CheckCsrKernel<<<GridOf(n, 128, sm_count), 128, 0, run.stream>>>(n, m_nnz, m_offsets, m_indices, kBadM, check);
    run.Launched("check M");
  }
  unsigned long long bad = 0;
  run.Ok(cudaMemcpyAsync(&bad, check, sizeof(bad), cudaMemcpyDeviceToHost, run.stream), "status readback");
  run.Ok(cudaStreamSynchronize(run.stream), "status readback");
  if (run.failed) return -1;
  if (bad != 0) {
    const char* which = (bad & kBadA) && (bad & kBadM) ? "A and M" : ((bad & kBadA) ? "A" : "M");
    SetError(error, error_capacity, "malformed CSR input (%s): offsets must run from 0 to nnz without decreasing "
             "and column indices must lie in [0, n)", which);
    return -1;
  }

  const int vec_grid = GridOf(n, 256, sm_count);

  // x0 = 0, r = b, z = M r, p = z
  run.Ok(cudaMemsetAsync(x, 0, sizeof(double) * n, run.stream), "clear x");
  run.Ok(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, run.stream), "r = b");
  run.Spmv(m_offsets, m_indices, m_values, r, z);
  run.Ok(cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, run.stream), "p = z");
  double r_r = run.Dot(r, r);
  const double b_norm = std::sqrt(r_r);
  double r_z = run.Dot(r, z);
  history[0] = 1.0;
  int64_t count = 1;
  int64_t result_status = 0;
  while (!run.failed && count < max_iterations && history[count - 1] > tolerance) {
    run.Spmv(a_offsets, a_indices, a_values, p, ap);
    const double den = run.Dot(p, ap);
    if (!std::isfinite(r_z) || !std::isfinite(den) || r_z == 0.0 || den == 0.0) {
      result_status = 2;
      break;
    }
    const double alpha = r_z / den;
    if (!std::isfinite(alpha)) {
      result_status = 2;
      break;
    }
    double beta = r_z;
    if (!run.failed) {
      NoAllocStepKernel<<<vec_grid, 256, 0, run.stream>>>(n, alpha, p, ap, x, r);
      run.Launched("step");
    }
    r_r = run.Dot(r, r);
    double residual = std::sqrt(r_r) / b_norm;
    const bool converged_refresh = residual <= tolerance;
    const bool periodic_refresh = refresh_period > 0 && count % refresh_period == 0;
    if (converged_refresh || periodic_refresh) {
      run.Spmv(a_offsets, a_indices, a_values, x, ap);
      if (!run.failed) {
        NoAllocResidualKernel<<<vec_grid, 256, 0, run.stream>>>(n, b, ap, r);
        run.Launched("true residual");
      }
      r_r = run.Dot(r, r);
      residual = std::sqrt(r_r) / b_norm;
    }
    run.Spmv(m_offsets, m_indices, m_values, r, z);
    r_z = run.Dot(r, z);
    beta = converged_refresh ? 0.0 : r_z / beta;
    history[count] = residual;
    ++count;
    if (!std::isfinite(residual)) {
      result_status = 3;
      break;
    }
    if (!std::isfinite(beta)) {
      result_status = 2;
      break;
    }
    if (!run.failed) {
      NoAllocDirectionKernel<<<vec_grid, 256, 0, run.stream>>>(n, beta, z, p);
      run.Launched("direction");
    }
  }
  // the last history entry is the true relative residual ||b - A x|| / ||b||
  run.Spmv(a_offsets, a_indices, a_values, x, ap);
  if (!run.failed) {
    NoAllocResidualKernel<<<vec_grid, 256, 0, run.stream>>>(n, b, ap, r);
    run.Launched("true residual");
  }
  history[count - 1] = std::sqrt(run.Dot(r, r)) / b_norm;
  run.Ok(cudaStreamSynchronize(run.stream), "final synchronise");
  if (run.failed) return -1;
  if (!std::isfinite(history[count - 1])) {
    result_status = 3;
  } else if (history[count - 1] <= tolerance) {
    result_status = 1;
  }
  if (status != nullptr) *status = result_status;
  return count;
}
