#pragma once
// Device solver for the five SPAI methods.  One Solver owns every matrix of
// the iteration in HBM (A and its row-compressed copy, M, R, Z, P, AP, AZ,
// Tmp, Q) and runs the reference's control flow with device kernels; the
// host only reads back the global scalars each iteration needs for its
// branch decisions (step lengths, convergence, sizes of new patterns).
//
// Global reductions use the device's canonical order: sequential inside a
// column (as Eigen sums a column), then the fixed 4096-wide tree across
// columns.  The CPU oracle reproduces that order bit for bit.

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/methods_c_api.h"
#include "device.cuh"
#include "ops.cuh"

namespace spai {

struct HostCsc {
  int64_t rows = 0;
  int64_t cols = 0;
  int64_t nnz = 0;
  const int64_t* ptr = nullptr;
  const int64_t* idx = nullptr;
  const double* val = nullptr;
};

enum class Method : int64_t {
  kGlobalCg = 0,
  kGlobalMr = 1,
  kGlobalLomr = 2,
  kInnerOuterMr = 3,
  kInnerOuterLomr = 4,
};

struct SolveOptions {
  Method method = Method::kGlobalMr;
  int64_t max_iterations = 100;
  double tolerance = 1e-9;
  double max_density = 0.03;
  bool dropping = true;
  int64_t inner_iterations = 2;
  int64_t topk = 0;       // 0: reference global budget; K > 0: per-column top-K by magnitude
  int precision = 0;      // 0: FP64 storage, 1: FP32 storage with FP64 reductions
  // 0: the device order -- sequential inside a column, then the fixed
  // 4096-wide tree across columns.  1: the reference's order -- columns in
  // min(n, num_threads) batches (methods_common.cpp:78-103,135-136), each
  // global sum sequential through a batch's columns in storage order, then
  // over the batches -- which reproduces the reference's recorded histories.
  int summation = 0;
  int64_t num_threads = 1;
};

// M on the host in the arrays the C ABI hands out (new[], released by
// free_mem), so a Result takes them over without a copy.
struct SolveOutput {
  int64_t rows = 0;
  int64_t cols = 0;
  int64_t nnz = 0;
  std::unique_ptr<int64_t[]> ptr;  // cols + 1
  std::unique_ptr<int64_t[]> idx;  // nnz
  std::unique_ptr<double[]> val;   // nnz
  std::vector<SingleIterationData> history;
  int64_t iterations = 0;
  bool converged = false;

  void Allocate(int64_t r, int64_t c, int64_t count) {
    rows = r;
    cols = c;
    nnz = count;
    ptr.reset(new int64_t[c + 1]);
    idx.reset(new int64_t[count]);
    val.reset(new double[count]);
  }
};

struct IterationTimes {
  double setup_ms = 0.0;
  double iterate_ms = 0.0;
};

// A canonical n x n CSC in device memory (offsets from 0 to nnz, rows
// strictly increasing in every column), int64 indices and FP64 values.
struct DeviceCscInput {
  int64_t n = 0;
  int64_t nnz = 0;
  const int64_t* col_offsets = nullptr;
  const int64_t* row_indices = nullptr;
  const double* values = nullptr;
};

class SolverBase {
 public:
  virtual ~SolverBase() = default;
  // Host-to-device upload and one-time setup (row-compressed A, column norms,
  // preconditioner).  m0 / pr may be null (identity / diag(A)^-1).
  virtual void Upload(const HostCsc& a, const HostCsc* m0, const HostCsc* pr) = 0;
  // The same from device memory (checked on the device); Pr = diag(A)^-1.
  virtual void UploadDevice(const DeviceCscInput& a, const DeviceCscInput* m0) = 0;
  // Runs the method from M0; may be called repeatedly.
  virtual void Run() = 0;
  // Copies M (as FP64, int64 indices) and the history to the host.
  virtual void Download(SolveOutput& out) = 0;
  // Copies M into DEVICE arrays of n() + 1 (ptr) and m_nnz() (idx, val) entries (int64, FP64); synchronises.
  virtual void ExportMDevice(int64_t* ptr, int64_t* idx, double* val) = 0;
  // Copies M straight into host arrays of n() + 1 (ptr) and m_nnz() (idx, val) entries.
  virtual void DownloadM(int64_t* ptr, int64_t* idx, double* val) = 0;
  virtual const std::vector<SingleIterationData>& history() const = 0;
  virtual bool converged() const = 0;
  virtual int64_t iterations() const = 0;
  virtual int64_t m_nnz() const = 0;
  // Device CSR copy of the current M (rows as major), values widened to FP64
  // or kept in FP32 depending on want_fp32; used by the PCG evaluator.
  virtual void ExportMForPcg(void* csr_out, bool want_fp32) = 0;
  // Global MR on every diagonal block of the uploaded A on its own: block b
  // is rows and columns [offsets[b], offsets[b + 1]), with Pr = diag(A)^-1 and
  // per-column top-k or no dropping (the rules that stay inside a block).
  // Every launch covers all blocks; the step lengths, norms and stop rules
  // are per block.  outputs[b] gets block b's M (local indices) and history.
  virtual void RunMrBatched(const std::vector<int64_t>& offsets, std::vector<SolveOutput>& outputs) = 0;
  virtual const void* DeviceA() const = 0;  // DevCsc<double>* when precision == 0, else DevCsc<float>*
  virtual const void* DeviceA64() const = 0;  // DevCsc<double>* (always)
  virtual int64_t n() const = 0;
};

std::unique_ptr<SolverBase> MakeSolver(Ctx& ctx, const SolveOptions& options);

// Uploads a host CSC (int64 indices, f64 values, offsets rebased to start at
// 0) as DevCsc<T> (T = double or float); stage_* are scratch.  Synchronises.
template <class T>
void UploadCsc(Ctx& ctx, const HostCsc& h, DevCsc<T>& d, DevBuf<int64_t>& stage_idx, DevBuf<double>& stage_val);

// Validation shared by the C entry points (reference methods_c_api.cpp:16-40,
// methods_common.cpp:12-48); throws std::invalid_argument with the reference's messages.
HostCsc CheckedMatrix(const MatrixData& data);
// A canonical CSC in device memory -> out (int32 rows), checked on the device; throws with `name`.
void UploadCheckedDeviceCsc(Ctx& ctx, const DeviceCscInput& in, DevCsc<double>& out, const char* name);
void ValidateProblem(const HostCsc& a, const HostCsc* m0, const HostCsc* pr, const MethodParams& p);

}  // namespace spai
