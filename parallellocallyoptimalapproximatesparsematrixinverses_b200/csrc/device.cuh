#pragma once
// Device-side building blocks shared by every kernel file: error handling,
// stream-ordered buffers, the CSC/CSR layouts kept in HBM, and small helpers.
//
// HBM layout of a sparse matrix (column-compressed, like the reference's
// Eigen::SparseMatrix<double, ColMajor, int64_t>, include/methods.hpp:17):
//   ptr : int64[cols + 1]  column offsets (int64 so nnz may exceed 2^31)
//   idx : int32[nnz]       row indices, ascending inside each column
//   val : T[nnz]           T = double (FP64 mode) or float (mixed mode)
// Row indices are 32-bit because n < 2^31 is enforced at the boundary; this
// cuts index traffic by a third against the reference's int64.

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

namespace spai {

class CudaError : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

#define SPAI_CUDA(call)                                                                          \
  do {                                                                                           \
    const cudaError_t spai_err_ = (call);                                                        \
    if (spai_err_ != cudaSuccess) {                                                              \
      throw ::spai::CudaError(std::string("CUDA error: ") + cudaGetErrorString(spai_err_) +       \
                              " (" #call ") at " + __FILE__ + ":" + std::to_string(__LINE__));   \
    }                                                                                            \
  } while (0)

// Counts every kernel launch of the library (reported by spai_kernel_launches).
void CountLaunch();

// Makes `device` the calling thread's current device for a scope and
// restores the caller's device afterwards, so that an entry point neither
// depends on nor changes the caller's choice of device.
class DeviceScope {
 public:
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&previous_) != cudaSuccess) previous_ = -1;
    if (device != previous_) {
      SPAI_CUDA(cudaSetDevice(device));
      changed_ = previous_ >= 0;
    }
  }
  ~DeviceScope() {
    if (changed_) cudaSetDevice(previous_);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;

 private:
  int previous_ = -1;
  bool changed_ = false;
};

// Fault injection for tests (spai_inject_allocation_failure): true once,
// when the armed number of growing reservations has passed.
bool AllocationFailureInjected();

// Per-stream cache of released device blocks.  A block released on stream s
// is handed to the next allocation on s that fits it (at least the request,
// at most twice it): stream order makes the reuse safe without events, and
// the iteration loop, whose buffers recur at similar sizes every step, stops
// calling the allocator.  CacheFlush frees a stream's blocks; CacheRetire
// hands them to the next calls on the same device instead (both before the
// stream is destroyed).
void* CacheTake(cudaStream_t stream, size_t bytes, size_t* capacity_bytes);
void CacheGive(cudaStream_t stream, void* block, size_t bytes);
void CacheFlush(cudaStream_t stream);
// After `stream` has been synchronised: its blocks join a pool of idle blocks
// of `device` that later streams on the device take from before allocating.
void CacheRetire(cudaStream_t stream, int device);
// Records the device a context's stream belongs to (until CacheRetire), so
// that the stream only ever receives that device's idle blocks.
void CacheRegisterStream(cudaStream_t stream, int device);

#define SPAI_LAUNCH_CHECK()          \
  do {                               \
    ::spai::CountLaunch();           \
    SPAI_CUDA(cudaGetLastError());   \
  } while (0)

constexpr int kWarp = 32;

inline int64_t CeilDiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Grid size for a grid-stride kernel: enough CTAs to fill every SM several
// times, never more than the work needs.
int GridFor(int64_t work_items, int threads_per_block);

// Stream-ordered device buffer: blocks come from the per-stream cache above,
// else from the device's default memory pool (cudaMallocAsync).
template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { Swap(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      Release();
      Swap(o);
    }
    return *this;
  }
  ~DevBuf() { Release(); }

  // Ensures room for n elements; contents are not preserved on growth.
  void Reserve(size_t n, cudaStream_t stream) {
    if (n <= capacity_) {
      size_ = n;
      stream_ = stream;
      return;
    }
    if (AllocationFailureInjected()) throw CudaError("CUDA error: injected allocation failure (out of memory)");
    Release();
    const size_t cap = n + n / 4 + 64;
    size_t got = 0;
    void* block = CacheTake(stream, cap * sizeof(T), &got);
    if (block != nullptr) {
      ptr_ = static_cast<T*>(block);
      capacity_ = got / sizeof(T);
    } else {
      SPAI_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ptr_), cap * sizeof(T), stream));
      capacity_ = cap;
    }
    size_ = n;
    stream_ = stream;
  }

  void Release() {
    if (ptr_ != nullptr) {
      CacheGive(stream_, ptr_, capacity_ * sizeof(T));
      ptr_ = nullptr;
    }
    capacity_ = 0;
    size_ = 0;
  }

  T* data() { return ptr_; }
  const T* data() const { return ptr_; }
  size_t size() const { return size_; }
  size_t capacity() const { return capacity_; }

  void Swap(DevBuf& o) noexcept {
    std::swap(ptr_, o.ptr_);
    std::swap(size_, o.size_);
    std::swap(capacity_, o.capacity_);
    std::swap(stream_, o.stream_);
  }

 private:
  T* ptr_ = nullptr;
  size_t size_ = 0;
  size_t capacity_ = 0;
  cudaStream_t stream_ = nullptr;
};

// Compressed sparse matrix in HBM.  As CSC: `major` = columns, idx = rows.
// The same struct holds a CSR copy (major = rows, idx = columns).
template <class T>
struct DevCsc {
  int64_t rows = 0;
  int64_t cols = 0;
  int64_t nnz = 0;
  DevBuf<int64_t> ptr;
  DevBuf<int32_t> idx;
  DevBuf<T> val;

  void Shape(int64_t r, int64_t c, cudaStream_t s) {
    rows = r;
    cols = c;
    ptr.Reserve(static_cast<size_t>(c + 1), s);
  }
  void ReserveNnz(int64_t count, cudaStream_t s) {
    nnz = count;
    idx.Reserve(static_cast<size_t>(count > 0 ? count : 1), s);
    val.Reserve(static_cast<size_t>(count > 0 ? count : 1), s);
  }
  void Swap(DevCsc& o) noexcept {
    std::swap(rows, o.rows);
    std::swap(cols, o.cols);
    std::swap(nnz, o.nnz);
    ptr.Swap(o.ptr);
    idx.Swap(o.idx);
    val.Swap(o.val);
  }
};

// Kernel-side view of a compressed matrix.
template <class T>
struct CscView {
  int64_t rows;
  int64_t cols;
  const int64_t* __restrict__ ptr;
  const int32_t* __restrict__ idx;
  const T* __restrict__ val;
};

template <class T>
inline CscView<T> View(const DevCsc<T>& m) {
  return CscView<T>{m.rows, m.cols, m.ptr.data(), m.idx.data(), m.val.data()};
}

// Plain IEEE operations that the compiler may not fuse into an FMA, so every
// product and sum rounds exactly like the reference's x86-64 build.
__device__ __forceinline__ double Mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double Add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float Mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float Add(float a, float b) { return __fadd_rn(a, b); }

}  // namespace spai
