// C-ABI entry points of libspai_b200.so: the reference's five methods and
// free_mem (include/methods_c_api.h), plus the extensions of spai_b200.h.
// Every entry point converts exceptions into the reference's error
// convention; nothing throws across the boundary.

#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

// cod2x2.cuh first: its arithmetic helpers must not see device.cuh's overloads
#include "cod2x2.cuh"
#include "../../include/methods_c_api.h"
#include "../../include/spai_b200.h"
#include "adjoint.cuh"
#include "device.cuh"
#include "ops.cuh"
#include "pcg.cuh"
#include "profile.cuh"
#include "mr_fused.cuh"
#include "solver.cuh"

namespace spai {

namespace {
std::atomic<int64_t> g_launches{0};
std::atomic<int64_t> g_fail_after{-1};
}  // namespace

void CountLaunch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
// Kernel nodes executed by a graph launch.
void CountLaunches(int64_t count) { g_launches.fetch_add(count, std::memory_order_relaxed); }

bool AllocationFailureInjected() {
  if (g_fail_after.load(std::memory_order_relaxed) < 0) return false;
  // the reservation that brings the count to zero fails, then the hook disarms
  return g_fail_after.fetch_sub(1, std::memory_order_relaxed) == 0;
}

namespace {

void CopyError(const std::string& message, char* out, int64_t capacity) {
  if (out == nullptr || capacity <= 0) return;
  const size_t n = std::min<size_t>(message.size(), static_cast<size_t>(capacity - 1));
  std::memcpy(out, message.data(), n);
  out[n] = '\0';
}

Result ErrorResult(const std::string& message) {
  Result out{};
  out.error_message = new char[message.size() + 1];
  std::memcpy(out.error_message, message.c_str(), message.size() + 1);
  return out;
}

// GetSuccessResult (methods_c_api.cpp:66-114): host arrays allocated with
// new[]; M's arrays are taken over from the SolveOutput.
Result SuccessResult(SolveOutput&& s) {
  std::unique_ptr<SingleIterationData[]> hist(new SingleIterationData[s.history.size()]);
  for (size_t i = 0; i < s.history.size(); ++i) hist[i] = s.history[i];
  Result out{};
  out.rows = s.rows;
  out.cols = s.cols;
  out.nnz = s.nnz;
  out.iterations = s.iterations;
  out.converged = s.converged ? 1 : 0;
  out.history_size = static_cast<int64_t>(s.history.size());
  out.col_offsets = s.ptr.release();
  out.row_indices = s.idx.release();
  out.values = s.val.release();
  out.history = hist.release();
  return out;
}

// The same Result, filled from the device without an intermediate host copy.
Result SolverResult(SolverBase& solver) {
  const std::vector<SingleIterationData>& history = solver.history();
  const int64_t n = solver.n();
  const int64_t nnz = solver.m_nnz();
  std::unique_ptr<int64_t[]> ptr(new int64_t[n + 1]);
  std::unique_ptr<int64_t[]> idx(new int64_t[nnz]);
  std::unique_ptr<double[]> val(new double[nnz]);
  std::unique_ptr<SingleIterationData[]> hist(new SingleIterationData[history.size()]);
  solver.DownloadM(ptr.get(), idx.get(), val.get());
  for (size_t i = 0; i < history.size(); ++i) hist[i] = history[i];
  Result out{};
  out.rows = n;
  out.cols = n;
  out.nnz = nnz;
  out.iterations = solver.iterations();
  out.converged = solver.converged() ? 1 : 0;
  out.history_size = static_cast<int64_t>(history.size());
  out.col_offsets = ptr.release();
  out.row_indices = idx.release();
  out.values = val.release();
  out.history = hist.release();
  return out;
}

int ResolveDevice(int64_t requested) {
  int count = 0;
  const cudaError_t err = cudaGetDeviceCount(&count);
  if (err != cudaSuccess || count == 0) {
    throw CudaError("no CUDA device is available to libspai_b200 (" + std::string(cudaGetErrorString(err)) + ")");
  }
  if (requested < 0) {
    int current = 0;
    SPAI_CUDA(cudaGetDevice(&current));
    return current;
  }
  if (requested >= count) throw std::invalid_argument("device ordinal out of range");
  return static_cast<int>(requested);
}

struct CtxGuard {
  DeviceScope scope;  // constructed first, restored last: the caller keeps its current device
  Ctx ctx;
  explicit CtxGuard(int device) : scope(device) {
    try {
      ctx.Init(device);
    } catch (...) {
      ctx.Destroy();  // what Init created so far
      throw;
    }
  }
  ~CtxGuard() { ctx.Destroy(); }
};

struct Inputs {
  HostCsc a;
  HostCsc m0;
  HostCsc pr;
  bool has_m0 = false;
  bool has_pr = false;
};

// The run options from the reference's MethodParams and the extension
// knobs (the matrices are checked by the callers).
SolveOptions ParseOptions(int64_t method, const MethodParams& params, const SpaiExtParams* ext) {
  if (method < 0 || method > 4) throw std::invalid_argument("unknown method id");
  if (method >= 3 && params.inner_iterations <= 0) throw std::invalid_argument("inner_iterations must be positive");
  SolveOptions opt;
  opt.method = static_cast<Method>(method);
  opt.max_iterations = params.max_iterations;
  opt.tolerance = params.tolerance;
  opt.max_density = params.max_density;
  opt.dropping = params.enable_dropping != 0;
  opt.inner_iterations = params.inner_iterations;
  opt.num_threads = params.num_threads;
  // Without extension knobs (the five methods_c_api.h entry points, or ext ==
  // NULL) a run is the reference's: FP64, global budget, and its summation
  // order over min(n, num_threads) column batches, so the drop-in returns the
  // reference's bits.
  opt.summation = 1;
  if (ext != nullptr) {
    if (ext->precision != 0 && ext->precision != 1) throw std::invalid_argument("precision must be 0 (FP64) or 1 (mixed)");
    if (ext->topk_per_column < 0) throw std::invalid_argument("topk_per_column must be non-negative");
    if (ext->summation_order != 0 && ext->summation_order != 1) {
      throw std::invalid_argument("summation_order must be 0 (device tree) or 1 (the reference's batches)");
    }
    opt.precision = static_cast<int>(ext->precision);
    opt.topk = ext->topk_per_column;
    opt.summation = static_cast<int>(ext->summation_order);
  }
  return opt;
}

SolveOptions CheckInputs(int64_t method, const MatrixData& A, const MatrixData& M0, const MatrixData& Pr,
                         const MethodParams& params, const SpaiExtParams* ext, Inputs& in) {
  if (method < 0 || method > 4) throw std::invalid_argument("unknown method id");
  in.a = CheckedMatrix(A);
  in.has_m0 = params.use_initial_m != 0;
  if (in.has_m0) in.m0 = CheckedMatrix(M0);
  in.has_pr = params.use_preconditioner != 0;
  if (in.has_pr) in.pr = CheckedMatrix(Pr);
  const SolveOptions opt = ParseOptions(method, params, ext);
  ValidateProblem(in.a, in.has_m0 ? &in.m0 : nullptr, in.has_pr ? &in.pr : nullptr, params);
  return opt;
}

Result RunMethod(int64_t method, MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params,
                 const SpaiExtParams* ext) {
  try {
    Inputs in;
    const SolveOptions opt = CheckInputs(method, A, M0, Pr, params, ext, in);
    CtxGuard guard(ResolveDevice(ext != nullptr ? ext->device : -1));
    auto solver = MakeSolver(guard.ctx, opt);
    solver->Upload(in.a, in.has_m0 ? &in.m0 : nullptr, in.has_pr ? &in.pr : nullptr);
    solver->Run();
    return SolverResult(*solver);
  } catch (const std::exception& ex) {
    return ErrorResult(ex.what());
  } catch (...) {
    return ErrorResult("Unknown failure.");
  }
}

// dst[i] = src[i] as int32; *bad = 1 when an index is outside [0, limit).
__global__ void NarrowCheckedKernel(const int64_t* __restrict__ src, int32_t* __restrict__ dst, int64_t n,
                                    int64_t limit, int32_t* __restrict__ bad) {
  bool out_of_range = false;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t v = src[i];
    out_of_range |= v < 0 || v >= limit;
    dst[i] = static_cast<int32_t>(v);
  }
  if (__any_sync(0xffffffffu, out_of_range) && (threadIdx.x & 31) == 0) atomicOr(bad, 1);
}

// Host CSR (int64) -> device row-compressed DevCsc (rows as major dimension).
// The offsets are checked on the host; the column indices go up as int64 and
// are narrowed and range-checked on the device.
template <class T>
void UploadCsr(Ctx& ctx, int64_t n, const double* values, const int64_t* indices, const int64_t* offsets,
               DevCsc<T>& out) {
  if (offsets[0] != 0) throw std::invalid_argument("CSR offsets must start at 0");
  for (int64_t i = 0; i < n; ++i) {
    if (offsets[i] > offsets[i + 1]) throw std::invalid_argument("CSR offsets must be non-decreasing");
  }
  const int64_t nnz = offsets[n];
  out.Shape(n, n, ctx.stream);
  out.ReserveNnz(nnz, ctx.stream);
  SPAI_CUDA(cudaMemcpyAsync(out.ptr.data(), offsets, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, ctx.stream));
  if (nnz > 0) {
    DevBuf<int64_t> wide;
    wide.Reserve(static_cast<size_t>(nnz), ctx.stream);
    SPAI_CUDA(cudaMemcpyAsync(wide.data(), indices, sizeof(int64_t) * nnz, cudaMemcpyHostToDevice, ctx.stream));
    int32_t* bad = ctx.flags.data() + 3;
    SPAI_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), ctx.stream));
    NarrowCheckedKernel<<<GridFor(nnz, 256), 256, 0, ctx.stream>>>(wide.data(), out.idx.data(), nnz, n, bad);
    SPAI_LAUNCH_CHECK();
    SPAI_CUDA(cudaMemcpyAsync(ctx.host_flags + 3, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
    if constexpr (sizeof(T) == sizeof(double)) {
      SPAI_CUDA(cudaMemcpyAsync(out.val.data(), values, sizeof(double) * nnz, cudaMemcpyHostToDevice, ctx.stream));
    } else {
      DevBuf<double> stage;
      stage.Reserve(static_cast<size_t>(nnz), ctx.stream);
      SPAI_CUDA(cudaMemcpyAsync(stage.data(), values, sizeof(double) * nnz, cudaMemcpyHostToDevice, ctx.stream));
      ConvertValues<double, T>(ctx, stage.data(), out.val.data(), nnz);
      ctx.Sync();
    }
    ctx.Sync();
    if (ctx.host_flags[3] != 0) throw std::invalid_argument("CSR column index out of range");
  }
  ctx.Sync();
}

// (M + M^T) / 2 of a row- or column-compressed M, in place.
template <class T>
void SymmetricPart(Ctx& ctx, DevCsc<T>& m) {
  DevCsc<T> mt;
  Transpose(ctx, m, mt);
  Union(ctx, m, false, 1.0, mt, 1.0, m, UnionMode::kHalfSum);
}

void CheckPcgParams(int64_t n, const PcgParams& p) {
  if (p.symmetric_part != 0 && p.symmetric_part != 1) throw std::invalid_argument("symmetric_part must be 0 or 1");
  if (n <= 0 || p.max_iterations <= 0) throw std::invalid_argument("n, max_iterations and threads must be positive");
  if (!(p.tolerance >= 0.0)) throw std::invalid_argument("tolerance must be non-negative");
  if (p.m_precision != 0 && p.m_precision != 1) throw std::invalid_argument("m_precision must be 0 or 1");
  if (p.refresh_period < 0) throw std::invalid_argument("refresh_period must be non-negative");
  if (n > static_cast<int64_t>(INT32_MAX)) throw std::invalid_argument("n exceeds the 32-bit index range");
}

int64_t FinishPcg(const PcgResult& r, int64_t capacity, double* history, int64_t* status) {
  const int64_t count = static_cast<int64_t>(r.history.size());
  if (history != nullptr) {
    for (int64_t i = 0; i < count && i < capacity; ++i) history[i] = r.history[i];
  }
  if (status != nullptr) *status = r.status;
  return count;
}

// f(0) .. f(count - 1) on host threads (systems are independent); the error
// of the first failing system, in system order, is the one rethrown.
template <class F>
void ForEachSystem(int64_t count, F f) {
  const int64_t threads = std::min<int64_t>(count, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
  std::vector<std::exception_ptr> errors(static_cast<size_t>(count));
  std::atomic<int64_t> next{0};
  auto work = [&]() {
    for (int64_t b = next.fetch_add(1); b < count; b = next.fetch_add(1)) {
      try {
        f(b);
      } catch (...) {
        errors[b] = std::current_exception();
      }
    }
  };
  std::vector<std::thread> pool;
  for (int64_t t = 1; t < threads; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  for (const auto& e : errors) {
    if (e) std::rethrow_exception(e);
  }
}

// Uploads CSR M as params ask (FP64 or FP32, optionally its symmetric part)
// and runs PCG from x = 0 on the device vectors rhs -> x.
void PcgOnDevice(Ctx& ctx, int64_t n, const DevCsc<double>& a, const double* m_values, const int64_t* m_indices,
                 const int64_t* m_offsets, const PcgParams& params, const double* rhs, double* x,
                 PcgResult& result) {
  PcgOptions opt;
  opt.max_iterations = params.max_iterations;
  opt.tolerance = params.tolerance;
  opt.refresh_period = params.refresh_period;
  if (params.m_precision == 1) {
    DevCsc<float> m;
    UploadCsr(ctx, n, m_values, m_indices, m_offsets, m);
    if (params.symmetric_part) SymmetricPart(ctx, m);
    RunPcg(ctx, a, m, rhs, x, opt, result);
  } else {
    DevCsc<double> m;
    UploadCsr(ctx, n, m_values, m_indices, m_offsets, m);
    if (params.symmetric_part) SymmetricPart(ctx, m);
    RunPcg(ctx, a, m, rhs, x, opt, result);
  }
}


// CSR offsets in device memory: *bad |= 1 unless they start at 0, never
// decrease and end at nnz.
__global__ void CheckOffsetsKernel(const int64_t* __restrict__ offsets, int64_t n, int64_t nnz,
                                   int32_t* __restrict__ bad) {
  bool wrong = false;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = offsets[i];
    const int64_t e = offsets[i + 1];
    wrong |= e < b || (i == 0 && b != 0) || (i == n - 1 && e != nnz);
  }
  if (__any_sync(0xffffffffu, wrong) && (threadIdx.x & 31) == 0) atomicOr(bad, 1);
}

// Throws unless ptr is device (or managed) memory of `device`.
void CheckDevicePointer(const void* ptr, int64_t count, const char* name, int device) {
  if (count <= 0) return;
  if (ptr == nullptr) throw std::invalid_argument(std::string(name) + " must not be null");
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
    cudaGetLastError();
    throw std::invalid_argument(std::string(name) + " is not a pointer CUDA knows");
  }
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) {
    throw std::invalid_argument(std::string(name) + " must point to device memory");
  }
  if (attr.type == cudaMemoryTypeDevice && attr.device != device) {
    throw std::invalid_argument(std::string(name) + " lives on another device than the call's");
  }
}

// Throws when the byte ranges [a, a + a_bytes) and [b, b + b_bytes) overlap.
void CheckDisjoint(const void* a, size_t a_bytes, const void* b, size_t b_bytes, const char* what) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(a);
  const uintptr_t b0 = reinterpret_cast<uintptr_t>(b);
  if (a == nullptr || b == nullptr || a_bytes == 0 || b_bytes == 0) return;
  if (a0 < b0 + b_bytes && b0 < a0 + a_bytes) throw std::invalid_argument(what);
}

// Device CSR (int64 offsets and indices, FP64 values) -> device row-compressed
// DevCsc<T>: offsets and index range checked on the device, values converted
// to T.  The device form of UploadCsr.
template <class T>
void UploadCsrDevice(Ctx& ctx, int64_t n, int64_t nnz, const double* values, const int64_t* indices,
                     const int64_t* offsets, DevCsc<T>& out) {
  out.Shape(n, n, ctx.stream);
  out.ReserveNnz(nnz, ctx.stream);
  SPAI_CUDA(cudaMemcpyAsync(out.ptr.data(), offsets, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToDevice, ctx.stream));
  int32_t* bad = ctx.flags.data() + 3;
  SPAI_CUDA(cudaMemsetAsync(bad, 0, 2 * sizeof(int32_t), ctx.stream));
  CheckOffsetsKernel<<<GridFor(n, 256), 256, 0, ctx.stream>>>(offsets, n, nnz, bad + 1);
  SPAI_LAUNCH_CHECK();
  if (nnz > 0) {
    NarrowCheckedKernel<<<GridFor(nnz, 256), 256, 0, ctx.stream>>>(indices, out.idx.data(), nnz, n, bad);
    SPAI_LAUNCH_CHECK();
    if constexpr (sizeof(T) == sizeof(double)) {
      SPAI_CUDA(cudaMemcpyAsync(out.val.data(), values, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, ctx.stream));
    } else {
      ConvertValues<double, T>(ctx, values, out.val.data(), nnz);
    }
  }
  SPAI_CUDA(cudaMemcpyAsync(ctx.host_flags + 3, bad, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.Sync();
  if (ctx.host_flags[4] != 0) throw std::invalid_argument("CSR offsets must start at 0, not decrease and end at nnz");
  if (ctx.host_flags[3] != 0) throw std::invalid_argument("CSR column index out of range");
}

// PcgOnDevice with M as device CSR arrays.
void PcgOnDeviceArrays(Ctx& ctx, int64_t n, const DevCsc<double>& a, int64_t m_nnz, const double* m_values,
                       const int64_t* m_indices, const int64_t* m_offsets, const PcgParams& params, const double* rhs,
                       double* x, PcgResult& result) {
  PcgOptions opt;
  opt.max_iterations = params.max_iterations;
  opt.tolerance = params.tolerance;
  opt.refresh_period = params.refresh_period;
  if (params.m_precision == 1) {
    DevCsc<float> m;
    UploadCsrDevice(ctx, n, m_nnz, m_values, m_indices, m_offsets, m);
    if (params.symmetric_part) SymmetricPart(ctx, m);
    RunPcg(ctx, a, m, rhs, x, opt, result);
  } else {
    DevCsc<double> m;
    UploadCsrDevice(ctx, n, m_nnz, m_values, m_indices, m_offsets, m);
    if (params.symmetric_part) SymmetricPart(ctx, m);
    RunPcg(ctx, a, m, rhs, x, opt, result);
  }
}

// The adjoint entry points index their gradients by stored entry, so they
// take canonical CSC only: offsets from 0 to nnz, rows strictly increasing
// inside every column (what methods.pyx:82-86 hands the reference).
void CheckCanonicalCsc(const HostCsc& h, const char* name) {
  if (h.ptr[0] != 0 || h.ptr[h.cols] != h.nnz) {
    throw std::invalid_argument(std::string(name) + ": column offsets must run from 0 to nnz");
  }
  for (int64_t j = 0; j < h.cols; ++j) {
    for (int64_t p = h.ptr[j] + 1; p < h.ptr[j + 1]; ++p) {
      if (h.idx[p] <= h.idx[p - 1]) {
        throw std::invalid_argument(std::string(name) + ": row indices must be strictly increasing in every column");
      }
    }
  }
}

}  // namespace
}  // namespace spai

struct SpaiSession {
  spai::Ctx ctx;
  std::unique_ptr<spai::SolverBase> solver;
  spai::SolveOptions options;
  int64_t n = 0;
  spai::DevBuf<double> b;
  spai::DevBuf<double> x;
  spai::DevCsc<double> a_rows;  // A as row-compressed FP64 for PCG
  spai::DevCsc<double> m64;
  spai::DevCsc<float> m32;
  bool has_rhs = false;
  bool has_a_rows = false;
  std::vector<SingleIterationData> history;
  ~SpaiSession() {
    solver.reset();
    b.Release();
    x.Release();
    a_rows = spai::DevCsc<double>();
    m64 = spai::DevCsc<double>();
    m32 = spai::DevCsc<float>();
    ctx.Destroy();
  }
};

extern "C" {

Result spai_global_cg(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params) {
  return spai::RunMethod(0, A, M0, Pr, params, nullptr);
}

Result spai_global_mr(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params) {
  return spai::RunMethod(1, A, M0, Pr, params, nullptr);
}

Result spai_global_lomr(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params) {
  return spai::RunMethod(2, A, M0, Pr, params, nullptr);
}

Result inner_outer_mr(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params) {
  return spai::RunMethod(3, A, M0, Pr, params, nullptr);
}

Result inner_outer_lomr(MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params) {
  return spai::RunMethod(4, A, M0, Pr, params, nullptr);
}

void free_mem(Result* result) {
  if (result == nullptr) return;
  delete[] result->col_offsets;
  delete[] result->row_indices;
  delete[] result->values;
  delete[] result->history;
  delete[] result->error_message;
  result->col_offsets = nullptr;
  result->row_indices = nullptr;
  result->values = nullptr;
  result->history = nullptr;
  result->error_message = nullptr;
}

void spai_inject_allocation_failure(int64_t after) { spai::g_fail_after.store(after, std::memory_order_relaxed); }

namespace spai {
namespace {
// The device's 2x2 minimum-norm solve (the Inner-Outer LOMR step) on `count` systems.
__global__ void Solve2x2Kernel(int64_t count, const double* __restrict__ gram, const double* __restrict__ rhs,
                               double* __restrict__ out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double m[4] = {gram[4 * i], gram[4 * i + 1], gram[4 * i + 2], gram[4 * i + 3]};
    double x[2] = {rhs[2 * i], rhs[2 * i + 1]};
    double y[2];
    SolveLeastSquares2x2(m, x, y);
    out[2 * i] = y[0];
    out[2 * i + 1] = y[1];
  }
}
}  // namespace
}  // namespace spai

int64_t spai_solve_2x2_device(int64_t count, const double* gram, const double* rhs, double* out, char* error,
                              int64_t error_capacity) {
  try {
    if (count <= 0 || gram == nullptr || rhs == nullptr || out == nullptr) {
      throw std::invalid_argument("count must be positive and every array given");
    }
    spai::CtxGuard guard(spai::ResolveDevice(-1));
    spai::Ctx& ctx = guard.ctx;
    spai::DevBuf<double> g, r, o;
    g.Reserve(static_cast<size_t>(4 * count), ctx.stream);
    r.Reserve(static_cast<size_t>(2 * count), ctx.stream);
    o.Reserve(static_cast<size_t>(2 * count), ctx.stream);
    SPAI_CUDA(cudaMemcpyAsync(g.data(), gram, sizeof(double) * 4 * count, cudaMemcpyHostToDevice, ctx.stream));
    SPAI_CUDA(cudaMemcpyAsync(r.data(), rhs, sizeof(double) * 2 * count, cudaMemcpyHostToDevice, ctx.stream));
    spai::Solve2x2Kernel<<<spai::GridFor(count, 128), 128, 0, ctx.stream>>>(count, g.data(), r.data(), o.data());
    SPAI_LAUNCH_CHECK();
    SPAI_CUDA(cudaMemcpyAsync(out, o.data(), sizeof(double) * 2 * count, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.Sync();
    return 0;
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

void spai_free_int64_array(int64_t* array) { delete[] array; }

void spai_free_double_array(double* array) { delete[] array; }

Result spai_run_ex(int64_t method, MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params,
                   const SpaiExtParams* ext) {
  return spai::RunMethod(method, A, M0, Pr, params, ext);
}

int64_t spai_pcg(int64_t n, const double* a_values, const int64_t* a_indices, const int64_t* a_offsets,
                 const double* m_values, const int64_t* m_indices, const int64_t* m_offsets, const double* b,
                 PcgParams params, double* history, int64_t* status, double* x_out, char* error,
                 int64_t error_capacity) {
  try {
    spai::CheckPcgParams(n, params);
    spai::CtxGuard guard(spai::ResolveDevice(params.device));
    spai::Ctx& ctx = guard.ctx;
    spai::DevCsc<double> a;
    spai::UploadCsr(ctx, n, a_values, a_indices, a_offsets, a);
    spai::DevBuf<double> bd;
    spai::DevBuf<double> xd;
    bd.Reserve(static_cast<size_t>(n), ctx.stream);
    xd.Reserve(static_cast<size_t>(n), ctx.stream);
    SPAI_CUDA(cudaMemcpyAsync(bd.data(), b, sizeof(double) * n, cudaMemcpyHostToDevice, ctx.stream));
    spai::PcgResult result;
    spai::PcgOnDevice(ctx, n, a, m_values, m_indices, m_offsets, params, bd.data(), xd.data(), result);
    if (x_out != nullptr) {
      SPAI_CUDA(cudaMemcpyAsync(x_out, xd.data(), sizeof(double) * n, cudaMemcpyDeviceToHost, ctx.stream));
    }
    ctx.Sync();
    return spai::FinishPcg(result, params.max_iterations, history, status);
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_mr_batched(int64_t count, const MatrixData* A, const MatrixData* M0, MethodParams params,
                        const SpaiExtParams* ext, Result* results, char* error, int64_t error_capacity) {
  try {
    if (count <= 0 || A == nullptr || results == nullptr) {
      throw std::invalid_argument("count must be positive and A, results non-null");
    }
    for (int64_t b = 0; b < count; ++b) results[b] = Result{};
    if (params.use_initial_m != 0 && M0 == nullptr) throw std::invalid_argument("use_initial_m is set but M0 is null");
    if (params.use_preconditioner != 0) {
      throw std::invalid_argument("batched runs use Pr = diag(A)^-1: use_preconditioner must be 0");
    }
    const int64_t topk = ext != nullptr ? ext->topk_per_column : 0;
    if (params.enable_dropping != 0 && topk <= 0) {
      throw std::invalid_argument(
          "batched runs drop per column only: set topk_per_column > 0 or enable_dropping = 0");
    }
    // validation per system, with the reference's messages (methods_c_api.cpp:16-40, methods_common.cpp:12-48)
    std::vector<spai::HostCsc> as(static_cast<size_t>(count));
    std::vector<spai::HostCsc> ms(static_cast<size_t>(count));
    const bool has_m0 = params.use_initial_m != 0;
    spai::ForEachSystem(count, [&](int64_t b) {
      as[b] = spai::CheckedMatrix(A[b]);
      if (has_m0) ms[b] = spai::CheckedMatrix(M0[b]);
      spai::ValidateProblem(as[b], has_m0 ? &ms[b] : nullptr, nullptr, params);
    });
    std::vector<int64_t> offsets(static_cast<size_t>(count + 1), 0);
    std::vector<int64_t> a_at(static_cast<size_t>(count + 1), 0);
    std::vector<int64_t> m_at(static_cast<size_t>(count + 1), 0);
    for (int64_t b = 0; b < count; ++b) {
      offsets[b + 1] = offsets[b] + as[b].cols;
      a_at[b + 1] = a_at[b] + (as[b].ptr[as[b].cols] - as[b].ptr[0]);
      if (has_m0) m_at[b + 1] = m_at[b] + (ms[b].ptr[ms[b].cols] - ms[b].ptr[0]);
    }
    const int64_t n = offsets[count];
    if (n > static_cast<int64_t>(INT32_MAX)) throw std::invalid_argument("the batch exceeds 2^31 - 1 rows in total");
    // the block-diagonal matrices, assembled once on the host: system b's
    // columns, rows shifted by its first column, into disjoint ranges
    struct Assembled {
      std::unique_ptr<int64_t[]> ptr;
      std::unique_ptr<int64_t[]> idx;
      std::unique_ptr<double[]> val;
    };
    auto assemble = [&](const std::vector<spai::HostCsc>& parts, const std::vector<int64_t>& at) {
      Assembled out;
      const int64_t nnz = at[count];
      out.ptr.reset(new int64_t[n + 1]);
      out.idx.reset(new int64_t[nnz > 0 ? nnz : 1]);
      out.val.reset(new double[nnz > 0 ? nnz : 1]);
      out.ptr[0] = 0;
      spai::ForEachSystem(count, [&](int64_t b) {
        const spai::HostCsc& h = parts[b];
        const int64_t base = h.ptr[0];
        for (int64_t j = 0; j < h.cols; ++j) out.ptr[offsets[b] + j + 1] = at[b] + (h.ptr[j + 1] - base);
        const int64_t count_b = h.ptr[h.cols] - base;
        for (int64_t q = 0; q < count_b; ++q) {
          out.idx[at[b] + q] = h.idx[base + q] + offsets[b];
          out.val[at[b] + q] = h.val[base + q];
        }
      });
      return out;
    };
    const Assembled big_a_arrays = assemble(as, a_at);
    spai::HostCsc big_a{n, n, a_at[count], big_a_arrays.ptr.get(), big_a_arrays.idx.get(), big_a_arrays.val.get()};
    Assembled big_m_arrays;
    spai::HostCsc big_m;
    if (has_m0) {
      big_m_arrays = assemble(ms, m_at);
      big_m = spai::HostCsc{n, n, m_at[count], big_m_arrays.ptr.get(), big_m_arrays.idx.get(), big_m_arrays.val.get()};
    }
    spai::SolveOptions opt;
    opt.method = spai::Method::kGlobalMr;
    opt.max_iterations = params.max_iterations;
    opt.tolerance = params.tolerance;
    opt.max_density = params.max_density;
    opt.dropping = params.enable_dropping != 0;
    if (ext != nullptr) {
      if (ext->precision != 0 && ext->precision != 1) throw std::invalid_argument("precision must be 0 (FP64) or 1 (mixed)");
      if (ext->summation_order != 0) throw std::invalid_argument("batched runs use the device summation order");
      opt.precision = static_cast<int>(ext->precision);
      opt.topk = topk;
    }
    spai::CtxGuard guard(spai::ResolveDevice(ext != nullptr ? ext->device : -1));
    auto solver = spai::MakeSolver(guard.ctx, opt);
    solver->Upload(big_a, params.use_initial_m != 0 ? &big_m : nullptr, nullptr);
    std::vector<spai::SolveOutput> outputs;
    solver->RunMrBatched(offsets, outputs);
    for (int64_t b = 0; b < count; ++b) results[b] = spai::SuccessResult(std::move(outputs[b]));
    return 0;
  } catch (const std::exception& ex) {
    if (results != nullptr) {
      for (int64_t b = 0; b < count; ++b) free_mem(&results[b]);
    }
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_pcg_adjoint(int64_t n, const double* a_values, const int64_t* a_indices, const int64_t* a_offsets,
                         const double* m_values, const int64_t* m_indices, const int64_t* m_offsets, const double* x,
                         const double* grad_x, PcgParams params, double* grad_b, double* grad_a, double* history,
                         int64_t* status, char* error, int64_t error_capacity) {
  try {
    spai::CheckPcgParams(n, params);
    if (grad_x == nullptr) throw std::invalid_argument("grad_x must not be null");
    if (grad_a != nullptr && x == nullptr) throw std::invalid_argument("x must not be null when grad_a is requested");
    spai::CtxGuard guard(spai::ResolveDevice(params.device));
    spai::Ctx& ctx = guard.ctx;
    spai::DevCsc<double> a;
    spai::UploadCsr(ctx, n, a_values, a_indices, a_offsets, a);
    spai::DevBuf<double> gd;
    spai::DevBuf<double> lambda;
    gd.Reserve(static_cast<size_t>(n), ctx.stream);
    lambda.Reserve(static_cast<size_t>(n), ctx.stream);
    SPAI_CUDA(cudaMemcpyAsync(gd.data(), grad_x, sizeof(double) * n, cudaMemcpyHostToDevice, ctx.stream));
    // A symmetric: A^T lambda = grad_x is the forward's own solve
    spai::PcgResult result;
    spai::PcgOnDevice(ctx, n, a, m_values, m_indices, m_offsets, params, gd.data(), lambda.data(), result);
    if (grad_b != nullptr) {
      SPAI_CUDA(cudaMemcpyAsync(grad_b, lambda.data(), sizeof(double) * n, cudaMemcpyDeviceToHost, ctx.stream));
    }
    spai::DevBuf<double> xd;
    spai::DevBuf<double> ga;
    if (grad_a != nullptr && a.nnz > 0) {
      xd.Reserve(static_cast<size_t>(n), ctx.stream);
      ga.Reserve(static_cast<size_t>(a.nnz), ctx.stream);
      SPAI_CUDA(cudaMemcpyAsync(xd.data(), x, sizeof(double) * n, cudaMemcpyHostToDevice, ctx.stream));
      spai::NegativeOuterOnRows(ctx, a, lambda.data(), xd.data(), ga.data());
      SPAI_CUDA(cudaMemcpyAsync(grad_a, ga.data(), sizeof(double) * a.nnz, cudaMemcpyDeviceToHost, ctx.stream));
    }
    ctx.Sync();
    return spai::FinishPcg(result, params.max_iterations, history, status);
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_residual_adjoint(MatrixData A, MatrixData M, int64_t device, double* loss, double* grad_m,
                              double* grad_a, char* error, int64_t error_capacity) {
  try {
    const spai::HostCsc a = spai::CheckedMatrix(A);
    const spai::HostCsc m = spai::CheckedMatrix(M);
    if (a.rows != a.cols || m.rows != a.rows || m.cols != a.cols) {
      throw std::invalid_argument("A and M must be square and of the same size");
    }
    spai::CheckCanonicalCsc(a, "A");
    spai::CheckCanonicalCsc(m, "M");
    if (loss == nullptr) throw std::invalid_argument("loss must not be null");
    spai::CtxGuard guard(spai::ResolveDevice(device));
    spai::Ctx& ctx = guard.ctx;
    spai::DevBuf<int64_t> stage_idx;
    spai::DevBuf<double> stage_val;
    spai::DevCsc<double> ad;
    spai::DevCsc<double> md;
    spai::UploadCsc(ctx, a, ad, stage_idx, stage_val);
    spai::UploadCsc(ctx, m, md, stage_idx, stage_val);
    spai::DevBuf<double> gm;
    spai::DevBuf<double> ga;
    if (grad_m != nullptr) gm.Reserve(static_cast<size_t>(m.nnz), ctx.stream);
    if (grad_a != nullptr) ga.Reserve(static_cast<size_t>(a.nnz), ctx.stream);
    spai::ResidualAdjoint(ctx, ad, md, loss, grad_m != nullptr ? gm.data() : nullptr,
                          grad_a != nullptr ? ga.data() : nullptr);
    if (grad_m != nullptr) {
      SPAI_CUDA(cudaMemcpyAsync(grad_m, gm.data(), sizeof(double) * m.nnz, cudaMemcpyDeviceToHost, ctx.stream));
    }
    if (grad_a != nullptr) {
      SPAI_CUDA(cudaMemcpyAsync(grad_a, ga.data(), sizeof(double) * a.nnz, cudaMemcpyDeviceToHost, ctx.stream));
    }
    ctx.Sync();
    return 0;
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_pcg_device(int64_t n, int64_t a_nnz, const double* a_values, const int64_t* a_indices,
                        const int64_t* a_offsets, int64_t m_nnz, const double* m_values, const int64_t* m_indices,
                        const int64_t* m_offsets, const double* b, PcgParams params, double* history, int64_t* status,
                        double* x, char* error, int64_t error_capacity) {
  try {
    spai::CheckPcgParams(n, params);
    if (a_nnz < 0 || m_nnz < 0) throw std::invalid_argument("nnz must be non-negative");
    const int device = spai::ResolveDevice(params.device);
    spai::DeviceScope scope(device);
    spai::CheckDevicePointer(a_offsets, n + 1, "A offsets", device);
    spai::CheckDevicePointer(a_indices, a_nnz, "A indices", device);
    spai::CheckDevicePointer(a_values, a_nnz, "A values", device);
    spai::CheckDevicePointer(m_offsets, n + 1, "M offsets", device);
    spai::CheckDevicePointer(m_indices, m_nnz, "M indices", device);
    spai::CheckDevicePointer(m_values, m_nnz, "M values", device);
    spai::CheckDevicePointer(b, n, "b", device);
    spai::CheckDevicePointer(x, n, "x", device);
    spai::CheckDisjoint(x, sizeof(double) * n, b, sizeof(double) * n, "x overlaps b: x must not alias any input");
    spai::CtxGuard guard(device);
    spai::Ctx& ctx = guard.ctx;
    spai::DevCsc<double> a;
    spai::UploadCsrDevice(ctx, n, a_nnz, a_values, a_indices, a_offsets, a);
    spai::PcgResult result;
    spai::PcgOnDeviceArrays(ctx, n, a, m_nnz, m_values, m_indices, m_offsets, params, b, x, result);
    ctx.Sync();
    return spai::FinishPcg(result, params.max_iterations, history, status);
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_pcg_adjoint_device(int64_t n, int64_t a_nnz, const double* a_values, const int64_t* a_indices,
                                const int64_t* a_offsets, int64_t m_nnz, const double* m_values,
                                const int64_t* m_indices, const int64_t* m_offsets, const double* x,
                                const double* grad_x, PcgParams params, double* grad_b, double* grad_a,
                                double* history, int64_t* status, char* error, int64_t error_capacity) {
  try {
    spai::CheckPcgParams(n, params);
    if (a_nnz < 0 || m_nnz < 0) throw std::invalid_argument("nnz must be non-negative");
    if (grad_x == nullptr) throw std::invalid_argument("grad_x must not be null");
    if (grad_a != nullptr && x == nullptr) throw std::invalid_argument("x must not be null when grad_a is requested");
    const int device = spai::ResolveDevice(params.device);
    spai::DeviceScope scope(device);
    spai::CheckDevicePointer(a_offsets, n + 1, "A offsets", device);
    spai::CheckDevicePointer(a_indices, a_nnz, "A indices", device);
    spai::CheckDevicePointer(a_values, a_nnz, "A values", device);
    spai::CheckDevicePointer(m_offsets, n + 1, "M offsets", device);
    spai::CheckDevicePointer(m_indices, m_nnz, "M indices", device);
    spai::CheckDevicePointer(m_values, m_nnz, "M values", device);
    spai::CheckDevicePointer(grad_x, n, "grad_x", device);
    if (x != nullptr) spai::CheckDevicePointer(x, n, "x", device);
    if (grad_b != nullptr) {
      spai::CheckDevicePointer(grad_b, n, "grad_b", device);
      spai::CheckDisjoint(grad_b, sizeof(double) * n, grad_x, sizeof(double) * n,
                          "grad_b overlaps grad_x: outputs must not alias any input");
      spai::CheckDisjoint(grad_b, sizeof(double) * n, x, sizeof(double) * n,
                          "grad_b overlaps x: outputs must not alias any input");
    }
    if (grad_a != nullptr) spai::CheckDevicePointer(grad_a, a_nnz, "grad_a", device);
    spai::CtxGuard guard(device);
    spai::Ctx& ctx = guard.ctx;
    spai::DevCsc<double> a;
    spai::UploadCsrDevice(ctx, n, a_nnz, a_values, a_indices, a_offsets, a);
    // A symmetric: A^T lambda = grad_x is the forward's own solve; lambda lands in grad_b when it is asked for
    spai::DevBuf<double> own;
    double* lambda = grad_b;
    if (lambda == nullptr) {
      own.Reserve(static_cast<size_t>(n), ctx.stream);
      lambda = own.data();
    }
    spai::PcgResult result;
    spai::PcgOnDeviceArrays(ctx, n, a, m_nnz, m_values, m_indices, m_offsets, params, grad_x, lambda, result);
    if (grad_a != nullptr && a.nnz > 0) spai::NegativeOuterOnRows(ctx, a, lambda, x, grad_a);
    ctx.Sync();
    return spai::FinishPcg(result, params.max_iterations, history, status);
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_residual_adjoint_device(int64_t n, int64_t a_nnz, const int64_t* a_col_offsets,
                                     const int64_t* a_row_indices, const double* a_values, int64_t m_nnz,
                                     const int64_t* m_col_offsets, const int64_t* m_row_indices,
                                     const double* m_values, int64_t device, double* loss, double* grad_m,
                                     double* grad_a, char* error, int64_t error_capacity) {
  try {
    if (n <= 0 || a_nnz < 0 || m_nnz < 0) throw std::invalid_argument("n must be positive and nnz non-negative");
    if (n > static_cast<int64_t>(INT32_MAX)) {
      throw std::invalid_argument("Sparse matrix dimensions exceed the 32-bit row index range of the device layout");
    }
    if (loss == nullptr) throw std::invalid_argument("loss must not be null");
    const int dev = spai::ResolveDevice(device);
    spai::DeviceScope scope(dev);
    spai::CheckDevicePointer(a_col_offsets, n + 1, "A col_offsets", dev);
    spai::CheckDevicePointer(a_row_indices, a_nnz, "A row_indices", dev);
    spai::CheckDevicePointer(a_values, a_nnz, "A values", dev);
    spai::CheckDevicePointer(m_col_offsets, n + 1, "M col_offsets", dev);
    spai::CheckDevicePointer(m_row_indices, m_nnz, "M row_indices", dev);
    spai::CheckDevicePointer(m_values, m_nnz, "M values", dev);
    if (grad_m != nullptr) spai::CheckDevicePointer(grad_m, m_nnz, "grad_m", dev);
    if (grad_a != nullptr) spai::CheckDevicePointer(grad_a, a_nnz, "grad_a", dev);
    spai::CtxGuard guard(dev);
    spai::Ctx& ctx = guard.ctx;
    spai::DevCsc<double> ad;
    spai::DevCsc<double> md;
    spai::UploadCheckedDeviceCsc(ctx, spai::DeviceCscInput{n, a_nnz, a_col_offsets, a_row_indices, a_values}, ad, "A");
    spai::UploadCheckedDeviceCsc(ctx, spai::DeviceCscInput{n, m_nnz, m_col_offsets, m_row_indices, m_values}, md, "M");
    spai::ResidualAdjoint(ctx, ad, md, loss, grad_m, grad_a);
    ctx.Sync();
    return 0;
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_matvec(int64_t n, const double* values, const int64_t* indices, const int64_t* offsets, const double* x,
                    double* y, int64_t device, char* error, int64_t error_capacity) {
  try {
    if (n <= 0) throw std::invalid_argument("Invalid matrix-vector dimensions or thread count");
    spai::CtxGuard guard(spai::ResolveDevice(device));
    spai::Ctx& ctx = guard.ctx;
    spai::DevCsc<double> a;
    spai::UploadCsr(ctx, n, values, indices, offsets, a);
    spai::DevBuf<double> xd;
    spai::DevBuf<double> yd;
    xd.Reserve(static_cast<size_t>(n), ctx.stream);
    yd.Reserve(static_cast<size_t>(n), ctx.stream);
    SPAI_CUDA(cudaMemcpyAsync(xd.data(), x, sizeof(double) * n, cudaMemcpyHostToDevice, ctx.stream));
    spai::Spmv(ctx, a, xd.data(), yd.data());
    SPAI_CUDA(cudaMemcpyAsync(y, yd.data(), sizeof(double) * n, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.Sync();
    return 0;
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

SpaiSession* spai_session_create(int64_t method, MatrixData A, MatrixData M0, MatrixData Pr, MethodParams params,
                                 const SpaiExtParams* ext, char* error, int64_t error_capacity) {
  SpaiSession* session = nullptr;
  try {
    spai::Inputs in;
    const spai::SolveOptions opt = spai::CheckInputs(method, A, M0, Pr, params, ext, in);
    const int device = spai::ResolveDevice(ext != nullptr ? ext->device : -1);
    spai::DeviceScope scope(device);
    session = new SpaiSession();
    session->ctx.Init(device);
    session->options = opt;
    session->n = in.a.cols;
    session->solver = spai::MakeSolver(session->ctx, opt);
    session->solver->Upload(in.a, in.has_m0 ? &in.m0 : nullptr, in.has_pr ? &in.pr : nullptr);
    return session;
  } catch (const std::exception& ex) {
    delete session;
    spai::CopyError(ex.what(), error, error_capacity);
    return nullptr;
  }
}

SpaiSession* spai_session_create_device(int64_t method, int64_t n, int64_t a_nnz, const int64_t* a_col_offsets,
                                        const int64_t* a_row_indices, const double* a_values, int64_t m0_nnz,
                                        const int64_t* m0_col_offsets, const int64_t* m0_row_indices,
                                        const double* m0_values, MethodParams params, const SpaiExtParams* ext,
                                        char* error, int64_t error_capacity) {
  SpaiSession* session = nullptr;
  try {
    if (method < 0 || method > 4) throw std::invalid_argument("unknown method id");
    // GetCompressedSparseMatrix (methods_c_api.cpp:16-40) on the sizes; the arrays are checked on the device
    if (n <= 0 || a_nnz <= 0) throw std::invalid_argument("Sparse matrix dimensions and nnz must be positive");
    if (params.use_initial_m != 0 && m0_nnz <= 0) {
      throw std::invalid_argument("Sparse matrix dimensions and nnz must be positive");
    }
    if (n > static_cast<int64_t>(INT32_MAX)) {
      throw std::invalid_argument("Sparse matrix dimensions exceed the 32-bit row index range of the device layout");
    }
    if (params.use_preconditioner != 0) {
      throw std::invalid_argument("device sessions use Pr = diag(A)^-1: use_preconditioner must be 0");
    }
    const spai::SolveOptions opt = spai::ParseOptions(method, params, ext);
    // ValidateProblem reads only the shapes
    spai::HostCsc shape_a;
    shape_a.rows = shape_a.cols = n;
    shape_a.nnz = a_nnz;
    spai::HostCsc shape_m = shape_a;
    shape_m.nnz = m0_nnz;
    spai::ValidateProblem(shape_a, params.use_initial_m != 0 ? &shape_m : nullptr, nullptr, params);
    const int device = spai::ResolveDevice(ext != nullptr ? ext->device : -1);
    spai::DeviceScope scope(device);
    auto check = [&](const void* ptr, size_t bytes, const char* name) {
      if (bytes == 0) return;
      cudaPointerAttributes attr{};
      if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
        cudaGetLastError();
        throw std::invalid_argument(std::string(name) + " is not a pointer CUDA knows");
      }
      if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) {
        throw std::invalid_argument(std::string(name) + " must point to device memory");
      }
      if (attr.type == cudaMemoryTypeDevice && attr.device != device) {
        throw std::invalid_argument(std::string(name) + " lives on another device than the session's");
      }
    };
    check(a_col_offsets, sizeof(int64_t) * (n + 1), "A col_offsets");
    check(a_row_indices, sizeof(int64_t) * a_nnz, "A row_indices");
    check(a_values, sizeof(double) * a_nnz, "A values");
    spai::DeviceCscInput a{n, a_nnz, a_col_offsets, a_row_indices, a_values};
    spai::DeviceCscInput m0{n, m0_nnz, m0_col_offsets, m0_row_indices, m0_values};
    if (params.use_initial_m != 0) {
      check(m0_col_offsets, sizeof(int64_t) * (n + 1), "M0 col_offsets");
      check(m0_row_indices, sizeof(int64_t) * m0_nnz, "M0 row_indices");
      check(m0_values, sizeof(double) * m0_nnz, "M0 values");
    }
    session = new SpaiSession();
    session->ctx.Init(device);
    session->options = opt;
    session->n = n;
    session->solver = spai::MakeSolver(session->ctx, opt);
    session->solver->UploadDevice(a, params.use_initial_m != 0 ? &m0 : nullptr);
    return session;
  } catch (const std::exception& ex) {
    delete session;
    spai::CopyError(ex.what(), error, error_capacity);
    return nullptr;
  }
}

int64_t spai_session_result_device(SpaiSession* session, int64_t* col_offsets, int64_t* row_indices, double* values,
                                   int64_t capacity, char* error, int64_t error_capacity) {
  try {
    if (session == nullptr) throw std::invalid_argument("null session");
    spai::DeviceScope scope(session->ctx.device);
    const int64_t nnz = session->solver->m_nnz();
    if (capacity < nnz) throw std::invalid_argument("capacity is smaller than nnz(M)");
    session->solver->ExportMDevice(col_offsets, row_indices, values);
    return nnz;
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_session_run(SpaiSession* session, int64_t* iterations, int64_t* converged, int64_t* nnz_m, char* error,
                         int64_t error_capacity) {
  try {
    if (session == nullptr) throw std::invalid_argument("null session");
    spai::DeviceScope scope(session->ctx.device);
    session->solver->Run();
    if (iterations != nullptr) *iterations = session->solver->iterations();
    if (nnz_m != nullptr) *nnz_m = session->solver->m_nnz();
    if (converged != nullptr) *converged = session->solver->converged() ? 1 : 0;
    session->history.clear();
    return 0;
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_session_history(SpaiSession* session, SingleIterationData* out, int64_t capacity) {
  if (session == nullptr) return 0;
  try {
    const std::vector<SingleIterationData>& history = session->solver->history();
    const int64_t count = static_cast<int64_t>(history.size());
    for (int64_t i = 0; i < count && i < capacity; ++i) out[i] = history[i];
    return count;
  } catch (...) {
    return 0;
  }
}

Result spai_session_result(SpaiSession* session) {
  try {
    if (session == nullptr) throw std::invalid_argument("null session");
    spai::DeviceScope scope(session->ctx.device);
    return spai::SolverResult(*session->solver);
  } catch (const std::exception& ex) {
    return spai::ErrorResult(ex.what());
  }
}

int64_t spai_session_set_rhs(SpaiSession* session, const double* b, char* error, int64_t error_capacity) {
  try {
    if (session == nullptr) throw std::invalid_argument("null session");
    spai::DeviceScope scope(session->ctx.device);
    const int64_t n = session->n;
    session->b.Reserve(static_cast<size_t>(n), session->ctx.stream);
    session->x.Reserve(static_cast<size_t>(n), session->ctx.stream);
    SPAI_CUDA(cudaMemcpyAsync(session->b.data(), b, sizeof(double) * n, cudaMemcpyHostToDevice, session->ctx.stream));
    session->ctx.Sync();
    session->has_rhs = true;
    if (!session->has_a_rows) {
      const auto* a64 = static_cast<const spai::DevCsc<double>*>(session->solver->DeviceA64());
      spai::Transpose(session->ctx, *a64, session->a_rows);
      session->has_a_rows = true;
    }
    return 0;
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

int64_t spai_session_pcg(SpaiSession* session, PcgParams params, double* history, int64_t* status, double* x_out,
                         char* error, int64_t error_capacity) {
  try {
    if (session == nullptr) throw std::invalid_argument("null session");
    spai::DeviceScope scope(session->ctx.device);
    if (!session->has_rhs) throw std::invalid_argument("spai_session_set_rhs must be called first");
    spai::CheckPcgParams(session->n, params);
    spai::PcgOptions opt;
    opt.max_iterations = params.max_iterations;
    opt.tolerance = params.tolerance;
    opt.refresh_period = params.refresh_period;
    spai::PcgResult result;
    if (params.m_precision == 1) {
      session->solver->ExportMForPcg(&session->m32, true);
      if (params.symmetric_part) spai::SymmetricPart(session->ctx, session->m32);
      spai::RunPcg(session->ctx, session->a_rows, session->m32, session->b.data(), session->x.data(), opt, result);
    } else {
      session->solver->ExportMForPcg(&session->m64, false);
      if (params.symmetric_part) spai::SymmetricPart(session->ctx, session->m64);
      spai::RunPcg(session->ctx, session->a_rows, session->m64, session->b.data(), session->x.data(), opt, result);
    }
    if (x_out != nullptr) {
      SPAI_CUDA(cudaMemcpyAsync(x_out, session->x.data(), sizeof(double) * session->n, cudaMemcpyDeviceToHost,
                                session->ctx.stream));
      session->ctx.Sync();
    }
    return spai::FinishPcg(result, params.max_iterations, history, status);
  } catch (const std::exception& ex) {
    spai::CopyError(ex.what(), error, error_capacity);
    return -1;
  }
}

void spai_session_destroy(SpaiSession* session) {
  if (session == nullptr) return;
  std::unique_ptr<spai::DeviceScope> scope;  // released after the session, restoring the caller's device
  try {
    scope.reset(new spai::DeviceScope(session->ctx.device));
  } catch (...) {
  }
  delete session;
}

void* spai_session_stream(SpaiSession* session) {
  return session != nullptr ? static_cast<void*>(session->ctx.stream) : nullptr;
}

void spai_profile_enable(int64_t on) { spai::prof::SetEnabled(on != 0); }

void spai_profile_reset(void) { spai::prof::Reset(); }

int64_t spai_profile_read(const char* name, double* ms, int64_t* launches, double* bytes) {
  double t = 0.0;
  double b = 0.0;
  int64_t c = 0;
  const bool seen = spai::prof::Read(name != nullptr ? name : "", &t, &c, &b);
  if (ms != nullptr) *ms = t;
  if (launches != nullptr) *launches = c;
  if (bytes != nullptr) *bytes = b;
  return seen ? 1 : 0;
}

int64_t spai_kernel_launches(void) { return spai::g_launches.load(); }

void spai_set_fused_mr(int64_t enabled) { spai::SetFusedMrEnabled(enabled != 0); }

}  // extern "C"
