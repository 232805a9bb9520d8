// PCG evaluator on sm_100a (reference methods_cython/backward_error.pyx:69-144).
//
// A whole solve is one CUDA graph launch: a prologue (x = 0, r = b, z = M r,
// p = z, ||b|| and <r, z>), a device-side WHILE loop whose body is one PCG
// iteration, and an epilogue (the true residual at exit).  Every scalar of
// the recurrence -- alpha, beta, the residual history, the stop tests and the
// status code -- lives in a device-resident PcgState and is decided by the
// kernels themselves, so the loop needs no host round trip; the body's last
// kernel sets the loop's condition.  The host reads the history back once,
// after the solve.
//
// Dot products keep the library's canonical tree (tree.cuh): each dot kernel
// runs one block per 4096-value chunk, its lanes forming the chunk sums in
// the tree's order, and the last block to finish folds the chunk sums with
// the same tree; the vector updates that precede a dot (x += alpha p and
// r -= alpha A p, r = b - A x) are fused into it.  The CPU oracle therefore
// reproduces every iterate bit for bit, as with the stepwise host loop this
// replaces.
//
// Graphs are built once per (device, n, precision of M) and kept: every
// pointer a solve uses is read from the PcgState, so a new solve only uploads
// that struct (about 250 bytes) before launching.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <vector>

#include "device.cuh"
#include "ops.cuh"
#include "pcg.cuh"
#include "profile.cuh"
#include "tree.cuh"

namespace spai {

void CountLaunches(int64_t count);

namespace {

// Device-resident state of one solve.  The host writes the inputs before the
// graph launch; the kernels own the recurrence fields.
struct PcgState {
  // A (FP64) and M (FP64 or FP32 values) as CSR with int32 column indices
  const int64_t* a_ptr;
  const int32_t* a_idx;
  const double* a_val;
  const int64_t* m_ptr;
  const int32_t* m_idx;
  const void* m_val;
  const double* b;
  double* x;
  double* r;
  double* z;
  double* p;
  double* ap;
  double* history;        // max_iterations entries
  double* partial;        // chunk sums: 2 * chunks
  unsigned int* arrive;   // blocks of the running dot kernel that are done
  int64_t n;
  int64_t chunks;
  int64_t max_iterations;
  int64_t refresh_period;
  double tolerance;
  int64_t body_limit;     // hard cap on loop-body executions
  // the recurrence (backward_error.pyx:100-143)
  double r_z;
  double alpha;
  double beta;
  double error;
  double b_norm;
  int64_t count;
  int64_t status;
  int64_t done;
  int64_t refresh;
  int64_t converged_refresh;
  int64_t bodies;         // loop-body executions so far
};

// Which product a SpMV launch forms.
enum SpmvWhat : int {
  kMrInit = 0,       // prologue: z = M r and p = z
  kApFromP = 1,      // loop: ap = A p
  kApFromX = 2,      // loop, on a refresh: ap = A x
  kMrLoop = 3,       // loop: z = M r
  kApFromXFinal = 4  // epilogue: ap = A x
};

// Which tree reduction (and fused update) a dot launch forms.
enum DotWhat : int {
  kInit = 0,     // r.r and r.z: ||b||, the first <r, z>, history[0]
  kDen = 1,      // p.ap: alpha, or a breakdown
  kStep = 2,     // x += alpha p, r -= alpha ap, then r.r: the residual and the refresh decision
  kRefresh = 3,  // r = b - ap, then r.r (on a refresh only)
  kRz = 4,       // r.z: beta, the history entry, the stop tests
  kFinal = 5     // r = b - ap, then r.r: the true residual at exit and the status
};

__global__ void PcgInitKernel(PcgState* __restrict__ s) {
  const int64_t n = s->n;
  const double* __restrict__ b = s->b;
  double* __restrict__ x = s->x;
  double* __restrict__ r = s->r;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    x[i] = 0.0;
    r[i] = b[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *s->arrive = 0u;
    s->bodies = 0;
  }
}

// One thread per row, entries in storage order (the reference's _row_dot).
template <class TV, int kWhat>
__global__ void __launch_bounds__(128) PcgSpmvKernel(PcgState* __restrict__ s) {
  if (kWhat == kApFromP || kWhat == kMrLoop) {
    if (s->done) return;
  }
  if (kWhat == kApFromX) {
    if (s->done || !s->refresh) return;
  }
  constexpr bool kUseM = kWhat == kMrInit || kWhat == kMrLoop;
  const int64_t* __restrict__ ptr = kUseM ? s->m_ptr : s->a_ptr;
  const int32_t* __restrict__ idx = kUseM ? s->m_idx : s->a_idx;
  const TV* __restrict__ val = kUseM ? static_cast<const TV*>(s->m_val) : reinterpret_cast<const TV*>(s->a_val);
  const double* __restrict__ in = kWhat == kApFromP ? s->p : (kUseM ? s->r : s->x);
  double* __restrict__ out = kUseM ? s->z : s->ap;
  double* __restrict__ copy = kWhat == kMrInit ? s->p : nullptr;
  const int64_t n = s->n;
  for (int64_t row = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; row < n;
       row += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double sum = 0.0;
    const int64_t end = ptr[row + 1];
    for (int64_t k = ptr[row]; k < end; ++k) sum = Add(sum, Mul(static_cast<double>(val[k]), in[idx[k]]));
    out[row] = sum;
    if (kWhat == kMrInit) copy[row] = sum;
  }
}

// One block of kTreeLanes threads per 4096-value chunk; the last block to
// finish folds the chunk sums and applies the recurrence (thread 0).
template <int kWhat>
__global__ void __launch_bounds__(kTreeLanes) PcgDotKernel(PcgState* __restrict__ s) {
  __shared__ double shared[kTreeLanes];
  __shared__ int last;
  if (kWhat == kDen || kWhat == kStep || kWhat == kRz) {
    if (s->done) return;
  }
  if (kWhat == kRefresh) {
    if (s->done || !s->refresh) return;
  }
  const int64_t n = s->n;
  const int t = threadIdx.x;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTreeChunk + t;
  double* __restrict__ r = s->r;
  const double* __restrict__ z = s->z;
  const double* __restrict__ p = s->p;
  const double* __restrict__ ap = s->ap;
  const double* __restrict__ b = s->b;
  double* __restrict__ x = s->x;
  const double alpha = kWhat == kStep ? s->alpha : 0.0;
  double acc0 = 0.0;
  double acc1 = 0.0;
#pragma unroll
  for (int m = 0; m < kTreeTerms; ++m) {
    const int64_t i = base + static_cast<int64_t>(kTreeLanes) * m;
    if (i < n) {
      if (kWhat == kInit) {
        const double ri = r[i];
        acc0 = Add(acc0, Mul(ri, ri));
        acc1 = Add(acc1, Mul(ri, z[i]));
      } else if (kWhat == kDen) {
        acc0 = Add(acc0, Mul(p[i], ap[i]));
      } else if (kWhat == kStep) {
        const double pi = p[i];
        x[i] = Add(x[i], Mul(alpha, pi));
        const double ri = __dsub_rn(r[i], Mul(alpha, ap[i]));
        r[i] = ri;
        acc0 = Add(acc0, Mul(ri, ri));
      } else if (kWhat == kRefresh || kWhat == kFinal) {
        const double ri = __dsub_rn(b[i], ap[i]);
        r[i] = ri;
        acc0 = Add(acc0, Mul(ri, ri));
      } else {  // kRz
        acc0 = Add(acc0, Mul(r[i], z[i]));
      }
    }
  }
  double total0 = TreeButterfly(acc0, shared);
  double total1 = kWhat == kInit ? TreeButterfly(acc1, shared) : 0.0;
  if (gridDim.x > 1) {
    const int64_t chunks = gridDim.x;
    if (t == 0) {
      s->partial[blockIdx.x] = total0;
      if (kWhat == kInit) s->partial[chunks + blockIdx.x] = total1;
      __threadfence();
      last = atomicAdd(s->arrive, 1u) == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    total0 = TreeLevel(s->partial, chunks, shared);
    if (kWhat == kInit) total1 = TreeLevel(s->partial + chunks, chunks, shared);
    if (t == 0) *s->arrive = 0u;
  }
  if (t != 0) return;
  const double tol = s->tolerance;
  if (kWhat == kInit) {
    s->b_norm = __dsqrt_rn(total0);
    s->r_z = total1;
    s->history[0] = 1.0;
    s->count = 1;
    s->status = 0;
    s->error = 1.0;
    s->refresh = 0;
    s->converged_refresh = 0;
    s->done = (1 < s->max_iterations && 1.0 > tol) ? 0 : 1;
  } else if (kWhat == kDen) {
    const double r_z = s->r_z;
    const double den = total0;
    if (!isfinite(r_z) || !isfinite(den) || r_z == 0.0 || den == 0.0) {
      s->status = 2;
      s->done = 1;
    } else {
      const double a = __ddiv_rn(r_z, den);
      if (!isfinite(a)) {
        s->status = 2;
        s->done = 1;
      } else {
        s->alpha = a;
      }
    }
  } else if (kWhat == kStep) {
    const double error = __ddiv_rn(__dsqrt_rn(total0), s->b_norm);
    const bool converged = error <= tol;
    const bool periodic = s->refresh_period > 0 && s->count % s->refresh_period == 0;
    s->error = error;
    s->converged_refresh = converged ? 1 : 0;
    s->refresh = (converged || periodic) ? 1 : 0;
  } else if (kWhat == kRefresh) {
    s->error = __ddiv_rn(__dsqrt_rn(total0), s->b_norm);
  } else if (kWhat == kRz) {
    const double r_z_new = total0;
    const double beta = s->converged_refresh ? 0.0 : __ddiv_rn(r_z_new, s->r_z);
    s->r_z = r_z_new;
    const double error = s->error;
    const int64_t count = s->count;
    s->history[count] = error;
    s->count = count + 1;
    if (!isfinite(error)) {
      s->status = 3;
      s->done = 1;
    } else if (!isfinite(beta)) {
      s->status = 2;
      s->done = 1;
    } else {
      s->beta = beta;
      if (!(count + 1 < s->max_iterations && error > tol)) s->done = 1;
    }
  } else {  // kFinal
    const double h = __ddiv_rn(__dsqrt_rn(total0), s->b_norm);
    s->history[s->count - 1] = h;
    if (!isfinite(h)) {
      s->status = 3;
    } else if (h <= tol) {
      s->status = 1;
    }
  }
}

// p = z + beta p, then the loop's condition for the next body execution.
__global__ void PcgDirectionKernel(PcgState* __restrict__ s, cudaGraphConditionalHandle loop) {
  const bool done = s->done != 0;
  if (!done) {
    const int64_t n = s->n;
    const double beta = s->beta;
    const double* __restrict__ z = s->z;
    double* __restrict__ p = s->p;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      p[i] = Add(z[i], Mul(beta, p[i]));
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int64_t bodies = s->bodies + 1;
    s->bodies = bodies;
    // the body count bounds the loop whatever the recurrence does
    cudaGraphSetConditional(loop, (!done && bodies < s->body_limit) ? 1u : 0u);
  }
}

// Kernel nodes of one graph: prologue, per body execution, epilogue.
constexpr int64_t kPrologueKernels = 3;
constexpr int64_t kBodyKernels = 8;
constexpr int64_t kEpilogueKernels = 2;

// One instantiated solve graph with its state and scratch; used by one solve at a time.
struct PcgGraph {
  int device = -1;
  int64_t n = 0;
  bool fp32_m = false;
  bool busy = false;
  PcgState* state = nullptr;       // device
  PcgState* host_state = nullptr;  // pinned
  double* partial = nullptr;
  unsigned int* arrive = nullptr;
  cudaGraphExec_t exec = nullptr;
};

std::mutex g_graph_mutex;
std::vector<std::unique_ptr<PcgGraph>> g_graphs;  // kept for the process lifetime

template <class TM>
void CaptureGraph(PcgGraph& g, int sm_count) {
  const int64_t n = g.n;
  const int64_t chunks = CeilDiv(n, kTreeChunk);
  const int64_t cap = static_cast<int64_t>(sm_count) * 16;
  const int spmv_grid = static_cast<int>(std::min<int64_t>(CeilDiv(n, 128), cap));
  const int vec_grid = static_cast<int>(std::min<int64_t>(CeilDiv(n, 256), cap));
  const unsigned dot_grid = static_cast<unsigned>(chunks);
  cudaStream_t main_stream = nullptr;
  cudaStream_t body_stream = nullptr;
  cudaGraph_t graph = nullptr;
  SPAI_CUDA(cudaStreamCreateWithFlags(&main_stream, cudaStreamNonBlocking));
  try {
    SPAI_CUDA(cudaStreamCreateWithFlags(&body_stream, cudaStreamNonBlocking));
    SPAI_CUDA(cudaStreamBeginCapture(main_stream, cudaStreamCaptureModeThreadLocal));
    PcgState* s = g.state;
    PcgInitKernel<<<vec_grid, 256, 0, main_stream>>>(s);
    PcgSpmvKernel<TM, kMrInit><<<spmv_grid, 128, 0, main_stream>>>(s);
    PcgDotKernel<kInit><<<dot_grid, kTreeLanes, 0, main_stream>>>(s);
    SPAI_CUDA(cudaGetLastError());
    cudaStreamCaptureStatus status;
    cudaGraph_t capture_graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t num_deps = 0;
    SPAI_CUDA(cudaStreamGetCaptureInfo(main_stream, &status, nullptr, &capture_graph, &deps, &num_deps));
    cudaGraphConditionalHandle loop;
    SPAI_CUDA(cudaGraphConditionalHandleCreate(&loop, capture_graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = loop;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t loop_node;
    SPAI_CUDA(cudaGraphAddNode(&loop_node, capture_graph, deps, num_deps, &params));
    SPAI_CUDA(cudaStreamUpdateCaptureDependencies(main_stream, &loop_node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = params.conditional.phGraph_out[0];
    SPAI_CUDA(cudaStreamBeginCaptureToGraph(body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    PcgSpmvKernel<double, kApFromP><<<spmv_grid, 128, 0, body_stream>>>(s);
    PcgDotKernel<kDen><<<dot_grid, kTreeLanes, 0, body_stream>>>(s);
    PcgDotKernel<kStep><<<dot_grid, kTreeLanes, 0, body_stream>>>(s);
    PcgSpmvKernel<double, kApFromX><<<spmv_grid, 128, 0, body_stream>>>(s);
    PcgDotKernel<kRefresh><<<dot_grid, kTreeLanes, 0, body_stream>>>(s);
    PcgSpmvKernel<TM, kMrLoop><<<spmv_grid, 128, 0, body_stream>>>(s);
    PcgDotKernel<kRz><<<dot_grid, kTreeLanes, 0, body_stream>>>(s);
    PcgDirectionKernel<<<vec_grid, 256, 0, body_stream>>>(s, loop);
    SPAI_CUDA(cudaGetLastError());
    cudaGraph_t body_out = nullptr;
    SPAI_CUDA(cudaStreamEndCapture(body_stream, &body_out));
    PcgSpmvKernel<double, kApFromXFinal><<<spmv_grid, 128, 0, main_stream>>>(s);
    PcgDotKernel<kFinal><<<dot_grid, kTreeLanes, 0, main_stream>>>(s);
    SPAI_CUDA(cudaGetLastError());
    SPAI_CUDA(cudaStreamEndCapture(main_stream, &graph));
    SPAI_CUDA(cudaGraphInstantiate(&g.exec, graph, 0));
  } catch (...) {
    cudaStreamCaptureStatus st;
    for (cudaStream_t stream : {body_stream, main_stream}) {
      if (stream != nullptr && cudaStreamIsCapturing(stream, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
        cudaGraph_t dropped = nullptr;
        cudaStreamEndCapture(stream, &dropped);
        if (dropped != nullptr && stream == main_stream) cudaGraphDestroy(dropped);
      }
    }
    if (graph != nullptr) cudaGraphDestroy(graph);
    if (body_stream != nullptr) cudaStreamDestroy(body_stream);
    cudaStreamDestroy(main_stream);
    cudaGetLastError();
    throw;
  }
  cudaGraphDestroy(graph);
  cudaStreamDestroy(body_stream);
  cudaStreamDestroy(main_stream);
}

// A free graph for (device, n, precision of M), built on first use.
template <class TM>
PcgGraph* AcquireGraph(int device, int64_t n, int sm_count) {
  const bool fp32 = sizeof(TM) == sizeof(float);
  {
    std::lock_guard<std::mutex> lock(g_graph_mutex);
    for (auto& g : g_graphs) {
      if (!g->busy && g->device == device && g->n == n && g->fp32_m == fp32) {
        g->busy = true;
        return g.get();
      }
    }
  }
  auto g = std::make_unique<PcgGraph>();
  g->device = device;
  g->n = n;
  g->fp32_m = fp32;
  g->busy = true;
  try {
    SPAI_CUDA(cudaMalloc(reinterpret_cast<void**>(&g->state), sizeof(PcgState)));
    SPAI_CUDA(cudaMallocHost(reinterpret_cast<void**>(&g->host_state), sizeof(PcgState)));
    SPAI_CUDA(cudaMalloc(reinterpret_cast<void**>(&g->partial), sizeof(double) * 2 * CeilDiv(n, kTreeChunk)));
    SPAI_CUDA(cudaMalloc(reinterpret_cast<void**>(&g->arrive), sizeof(unsigned int)));
    SPAI_CUDA(cudaMemset(g->arrive, 0, sizeof(unsigned int)));
    CaptureGraph<TM>(*g, sm_count);
  } catch (...) {
    if (g->exec != nullptr) cudaGraphExecDestroy(g->exec);
    if (g->state != nullptr) cudaFree(g->state);
    if (g->host_state != nullptr) cudaFreeHost(g->host_state);
    if (g->partial != nullptr) cudaFree(g->partial);
    if (g->arrive != nullptr) cudaFree(g->arrive);
    throw;
  }
  std::lock_guard<std::mutex> lock(g_graph_mutex);
  g_graphs.push_back(std::move(g));
  return g_graphs.back().get();
}

void ReleaseGraph(PcgGraph* g) {
  std::lock_guard<std::mutex> lock(g_graph_mutex);
  g->busy = false;
}

// One thread per row, entries in storage order (the reference's _row_dot).
template <class TM>
__global__ void SpmvKernel(CscView<TM> a, const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t row = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; row < a.cols;
       row += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int64_t k = a.ptr[row]; k < a.ptr[row + 1]; ++k) {
      s = Add(s, Mul(static_cast<double>(a.val[k]), x[a.idx[k]]));
    }
    y[row] = s;
  }
}

}  // namespace

template <class TM>
void Spmv(Ctx& ctx, const DevCsc<TM>& a_rows, const double* x, double* y) {
  // algorithmic bytes: the matrix once, x once, y written once
  const double bytes = static_cast<double>(a_rows.nnz) * (sizeof(TM) + sizeof(int32_t)) +
                       static_cast<double>(a_rows.cols + 1) * sizeof(int64_t) + 16.0 * static_cast<double>(a_rows.cols);
  prof::Scope scope(ctx.stream, "pcg_spmv", bytes);
  SpmvKernel<TM><<<GridFor(a_rows.cols, 128), 128, 0, ctx.stream>>>(View(a_rows), x, y);
  SPAI_LAUNCH_CHECK();
}

template <class TM>
void RunPcg(Ctx& ctx, const DevCsc<double>& a, const DevCsc<TM>& m, const double* b, double* x,
            const PcgOptions& opt, PcgResult& result) {
  const int64_t n = a.cols;
  if (n <= 0) throw std::invalid_argument("PCG needs n > 0");
  if (n > kTreeChunk * kTreeChunk) throw std::invalid_argument("PCG supports at most 4096^2 rows");
  if (opt.max_iterations <= 0) throw std::invalid_argument("max_iterations must be positive");
  DevBuf<double> r, z, p, ap, history;
  r.Reserve(static_cast<size_t>(n), ctx.stream);
  z.Reserve(static_cast<size_t>(n), ctx.stream);
  p.Reserve(static_cast<size_t>(n), ctx.stream);
  ap.Reserve(static_cast<size_t>(n), ctx.stream);
  history.Reserve(static_cast<size_t>(opt.max_iterations), ctx.stream);
  PcgGraph* g = AcquireGraph<TM>(ctx.device, n, ctx.sm_count);
  try {
    PcgState& h = *g->host_state;
    h = PcgState{};
    h.a_ptr = a.ptr.data();
    h.a_idx = a.idx.data();
    h.a_val = a.val.data();
    h.m_ptr = m.ptr.data();
    h.m_idx = m.idx.data();
    h.m_val = m.val.data();
    h.b = b;
    h.x = x;
    h.r = r.data();
    h.z = z.data();
    h.p = p.data();
    h.ap = ap.data();
    h.history = history.data();
    h.partial = g->partial;
    h.arrive = g->arrive;
    h.n = n;
    h.chunks = CeilDiv(n, kTreeChunk);
    h.max_iterations = opt.max_iterations;
    h.refresh_period = opt.refresh_period;
    h.tolerance = opt.tolerance;
    h.body_limit = opt.max_iterations + 2;
    SPAI_CUDA(cudaMemcpyAsync(g->state, g->host_state, sizeof(PcgState), cudaMemcpyHostToDevice, ctx.stream));
    {
      prof::Scope scope(ctx.stream, "pcg_solve", 0.0);
      SPAI_CUDA(cudaGraphLaunch(g->exec, ctx.stream));
    }
    SPAI_CUDA(cudaMemcpyAsync(g->host_state, g->state, sizeof(PcgState), cudaMemcpyDeviceToHost, ctx.stream));
    result.history.assign(static_cast<size_t>(opt.max_iterations), 0.0);
    SPAI_CUDA(cudaMemcpyAsync(result.history.data(), history.data(), sizeof(double) * opt.max_iterations,
                              cudaMemcpyDeviceToHost, ctx.stream));
    ctx.Sync();
    const int64_t count = h.count;
    if (count < 1 || count > opt.max_iterations) throw CudaError("PCG graph returned an invalid iteration count");
    result.history.resize(static_cast<size_t>(count));
    result.status = h.status;
    result.spmv_count = 2 + 3 * (count - 1);
    // algorithmic bytes of the solve: per iteration A and M once plus the vector traffic (17 n doubles)
    const double per_iteration = static_cast<double>(a.nnz) * 12.0 + static_cast<double>(m.nnz) * (sizeof(TM) + 4) +
                                 8.0 * 17.0 * static_cast<double>(n);
    prof::AddBytes("pcg_solve", per_iteration * static_cast<double>(count));
    CountLaunches(kPrologueKernels + kBodyKernels * h.bodies + kEpilogueKernels);
  } catch (...) {
    ReleaseGraph(g);
    throw;
  }
  ReleaseGraph(g);
}

template void RunPcg<double>(Ctx&, const DevCsc<double>&, const DevCsc<double>&, const double*, double*,
                             const PcgOptions&, PcgResult&);
template void RunPcg<float>(Ctx&, const DevCsc<double>&, const DevCsc<float>&, const double*, double*,
                            const PcgOptions&, PcgResult&);
template void Spmv<double>(Ctx&, const DevCsc<double>&, const double*, double*);
template void Spmv<float>(Ctx&, const DevCsc<float>&, const double*, double*);

}  // namespace spai
