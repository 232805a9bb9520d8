#ifndef SPAI_B200_H_
#define SPAI_B200_H_
/*
 * Extensions of the drop-in C ABI (methods_c_api.h) served by libspai_b200.so.
 * C-clean: every declaration is extern "C" with plain pointers and sizes.
 * The structs MatrixData / MethodParams / SingleIterationData / Result are
 * the ones of methods_c_api.h, repeated here under an include guard so C
 * callers can use this header alone.
 *
 * Errors: functions returning Result put the message in error_message (the
 * reference's convention, methods_c_api.cpp:59-64); the others return a
 * negative value and copy the message into the caller's `error` buffer.
 */
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as methods_c_api.h (reference include/methods_c_api.h:7-46). */
#ifndef SPAI_ABI_STRUCTS_DEFINED
#define SPAI_ABI_STRUCTS_DEFINED
struct MatrixData {
  int64_t rows;
  int64_t cols;
  int64_t nnz;
  const int64_t* col_offsets;
  const int64_t* row_indices;
  const double* values;
};
struct MethodParams {
  int64_t max_iterations;
  double tolerance;
  double max_density;
  int64_t enable_dropping;
  int64_t num_threads;
  int64_t use_initial_m;
  int64_t use_preconditioner;
  int64_t inner_iterations;
};
struct SingleIterationData {
  int64_t iteration;
  double residual_norm;
  double density_m;
  double density_direction;
};
struct Result {
  int64_t rows;
  int64_t cols;
  int64_t nnz;
  int64_t iterations;
  int64_t converged;
  int64_t history_size;
  int64_t* col_offsets;
  int64_t* row_indices;
  double* values;
  struct SingleIterationData* history;
  char* error_message;
};
#endif

/* The reference's five entry points and free_mem (reference
 * include/methods_c_api.h:48-58), repeated so that C callers can use this
 * header alone; identical redeclarations of methods_c_api.h's. */
struct Result spai_global_cg(struct MatrixData A, struct MatrixData M0, struct MatrixData Pr,
                             struct MethodParams params);
struct Result spai_global_mr(struct MatrixData A, struct MatrixData M0, struct MatrixData Pr,
                             struct MethodParams params);
struct Result spai_global_lomr(struct MatrixData A, struct MatrixData M0, struct MatrixData Pr,
                               struct MethodParams params);
struct Result inner_outer_mr(struct MatrixData A, struct MatrixData M0, struct MatrixData Pr,
                             struct MethodParams params);
struct Result inner_outer_lomr(struct MatrixData A, struct MatrixData M0, struct MatrixData Pr,
                               struct MethodParams params);
void free_mem(struct Result* result);

/* Precision and selection knobs that the reference's MethodParams lacks. */
typedef struct SpaiExtParams {
  int64_t precision;       /* 0: FP64 storage (bit-compatible with the reference's arithmetic order inside each
                              column); 1: FP32 storage of M, R, Z, P, A with FP64 reductions */
  int64_t topk_per_column; /* 0: the reference's global budget max(n, floor(max_density*n^2)) (dropping.cpp:122-224);
                              K > 0: keep at most K entries per column by magnitude (diagonal of M protected) */
  int64_t device;          /* CUDA device ordinal; -1: the calling thread's current device */
  int64_t summation_order; /* 0: the device order (sequential per column, then a fixed 4096-wide tree);
                              1: the reference's order (min(n, num_threads) column batches, each global sum
                              sequential through a batch, then over the batches; methods_common.cpp:78-103):
                              FP64 runs then reproduce the reference's own results bit for bit */
} SpaiExtParams;

/* Release one array of a Result (col_offsets / row_indices: int64; values:
 * double) on its own, for callers that keep the arrays beyond the Result
 * (set the Result's field to NULL before free_mem). */
void spai_free_int64_array(int64_t* array);
void spai_free_double_array(double* array);

/* Method ids for spai_run_ex / sessions. */
enum {
  SPAI_GLOBAL_CG = 0,
  SPAI_GLOBAL_MR = 1,
  SPAI_GLOBAL_LOMR = 2,
  SPAI_INNER_OUTER_MR = 3,
  SPAI_INNER_OUTER_LOMR = 4
};

/* One call of any method with the extension knobs; ext may be NULL (FP64,
 * global budget, current device and the reference's summation order: what the
 * five methods_c_api.h entry points run, bit for bit the reference's results).
 * Replaces the five reference entry points of methods_c_api.h:48-56 (same
 * inputs, same Result ownership via free_mem). */
struct Result spai_run_ex(int64_t method, struct MatrixData A, struct MatrixData M0, struct MatrixData Pr,
                          struct MethodParams params, const SpaiExtParams* ext);

/* Global MR on `count` independent systems in one batch: A[b] (and M0[b]
 * when params.use_initial_m) are the reference's MatrixData, each square.  On
 * the device the systems form one block-diagonal problem, so every kernel
 * launch covers the whole batch, while step lengths, norms, stop rules and
 * histories stay per system: results[b] is what spai_global_mr would return
 * for system b alone (same bits in FP64).  Pr is diag(A[b])^-1
 * (params.use_preconditioner must be 0) and dropping, when enabled, must be
 * per column (ext->topk_per_column > 0).  Returns 0 with `count` Results to
 * release with free_mem each, or -1 with `error` and every results[b] empty. */
int64_t spai_mr_batched(int64_t count, const struct MatrixData* A, const struct MatrixData* M0,
                        struct MethodParams params, const SpaiExtParams* ext, struct Result* results, char* error,
                        int64_t error_capacity);

typedef struct PcgParams {
  int64_t max_iterations; /* length limit of the history, initial entry included (backward_error.pyx:69-72) */
  double tolerance;       /* relative residual ||r|| / ||b|| */
  int64_t refresh_period; /* 0: the reference's refresh at convergence only; K > 0: also r = b - A x every K steps */
  int64_t m_precision;    /* 0: M applied in FP64; 1: M stored in FP32, vectors and dots in FP64 */
  int64_t device;         /* CUDA device ordinal; -1: current device */
  int64_t symmetric_part; /* 0: precondition with M as given (the reference); 1: with (M + M^T)/2, formed on the
                             device (PCG assumes a symmetric preconditioner; SPAI iterates are not symmetric) */
} PcgParams;

/* PCG with x0 = 0 on CSR A and CSR M (int64 indices), the device form of the
 * reference's methods_cython/backward_error.pyx:69-144 `pcg`.  history must
 * hold params.max_iterations doubles; returns the number of entries written
 * (history[0] = 1), sets *status to 0 (iteration limit), 1 (converged),
 * 2 (recurrence breakdown) or 3 (non-finite residual); x_out (n doubles) may
 * be NULL.  Returns -1 and fills `error` on invalid input or CUDA failure. */
int64_t spai_pcg(int64_t n, const double* a_values, const int64_t* a_indices, const int64_t* a_offsets,
                 const double* m_values, const int64_t* m_indices, const int64_t* m_offsets, const double* b,
                 PcgParams params, double* history, int64_t* status, double* x_out, char* error,
                 int64_t error_capacity);

/* PCG on DEVICE buffers that allocates no memory.  No counterpart in the
 * reference: it is spai_pcg (FP64 M, same arithmetic, same bits) for callers
 * that cannot let a library allocate -- a solver loop that has given the
 * device's memory to its own pool, or one that must not stall other streams
 * through cudaMalloc/cudaFree.
 *   A and M: CSR on the current device, int64 offsets (n + 1), int32 column
 *   indices and FP64 values (nnz each); b and x: n doubles on the device
 *   (x is overwritten, x0 = 0); history: max_iterations host doubles.
 *   stream: the cudaStream_t to run on (NULL: the default stream).
 * Work vectors live in a fixed device array inside the library (16 MiB), so
 * n is limited to 524,288 rows; larger n returns -1 with an error.  Every
 * call looks up the array's device address in the current context; the
 * first call on a device can load the library's device code there, so make
 * that first call before any stream capture on the device.  The call is
 * host-synchronous: it returns when the solve is done, and waits for the
 * stream about three times per iteration to read scalars back.  Calls that
 * overlap on one GPU share the array and race: serialise them per device.
 * Pointers are checked (device memory of the current device, long enough;
 * x must not overlap b, A or M), offsets and indices are checked on the
 * device.  Returns the number of history entries and sets *status as
 * spai_pcg does; -1 with `error` on invalid input or CUDA failure. */
int64_t spai_pcg_device_noalloc(int64_t n, int64_t a_nnz, const double* a_values, const int32_t* a_indices,
                                const int64_t* a_offsets, int64_t m_nnz, const double* m_values,
                                const int32_t* m_indices, const int64_t* m_offsets, const double* b, double* x,
                                int64_t max_iterations, double tolerance, int64_t refresh_period, void* stream,
                                double* history, int64_t* status, char* error, int64_t error_capacity);

/* ---- Adjoints (reverse mode).  No counterpart in the reference; they
 * differentiate what the reference computes. ---- */

/* f(A, M) = ||I - A M||_F^2 -- the square of the residual norm the reference
 * records (methods_common.cpp:112-122) -- and its gradient with respect to the
 * stored values of M and of A.  A and M: n x n CSC in the reference's
 * MatrixData, canonical (offsets from 0 to nnz, rows strictly increasing in
 * every column).  On return *loss = f and, unless NULL,
 *   grad_m[p] = -2 (A^T R)(i, j)  for M's stored entry p = (i, j)  (nnz(M) doubles),
 *   grad_a[q] = -2 (R M^T)(i, k)  for A's stored entry q = (i, k)  (nnz(A) doubles),
 * with R = I - A M; every product in FP64, its terms summed in ascending k.
 * device: CUDA ordinal, -1 for the current device.  Returns 0, or -1 with `error`. */
int64_t spai_residual_adjoint(struct MatrixData A, struct MatrixData M, int64_t device, double* loss,
                              double* grad_m, double* grad_a, char* error, int64_t error_capacity);

/* Reverse mode of spai_pcg (x = A^-1 b for symmetric positive definite CSR A):
 * given x (the forward solution, n doubles) and grad_x = dL/dx, solves
 * A lambda = grad_x with the forward's preconditioner and settings (the same
 * arithmetic as spai_pcg with b = grad_x) and writes, unless NULL,
 *   grad_b[i] = lambda_i                                   (n doubles),
 *   grad_a[q] = -(lambda_i * x_j) for A's CSR entry q = (i, j)  (nnz(A) doubles).
 * This is the implicit-function adjoint: the gradient of the exact solution
 * map, which the computed x approximates to the solve's tolerance.  history
 * (params.max_iterations doubles) may be NULL; returns the adjoint solve's
 * history length and sets *status as spai_pcg does, or -1 with `error`. */
int64_t spai_pcg_adjoint(int64_t n, const double* a_values, const int64_t* a_indices, const int64_t* a_offsets,
                         const double* m_values, const int64_t* m_indices, const int64_t* m_offsets, const double* x,
                         const double* grad_x, PcgParams params, double* grad_b, double* grad_a, double* history,
                         int64_t* status, char* error, int64_t error_capacity);

/* ---- The same, on arrays already in device memory ----
 * Device forms of spai_pcg, spai_pcg_adjoint and spai_residual_adjoint for
 * callers whose data live on the GPU (torch CUDA tensors): every array
 * argument is device (or managed) memory of the call's device, with the
 * layouts, checks, arithmetic and results of the host forms (so the bits are
 * the same); the offsets and indices are validated on the device.  history,
 * status and loss stay host pointers.  Outputs must not alias inputs.  The
 * calls run on the library's own stream and return after it has finished:
 * the caller finishes the work that produces the inputs first (e.g. synchronises
 * its stream).  Each names its nnz explicitly: a_nnz = a_offsets[n]. */
int64_t spai_pcg_device(int64_t n, int64_t a_nnz, const double* a_values, const int64_t* a_indices,
                        const int64_t* a_offsets, int64_t m_nnz, const double* m_values, const int64_t* m_indices,
                        const int64_t* m_offsets, const double* b, PcgParams params, double* history, int64_t* status,
                        double* x, char* error, int64_t error_capacity);
int64_t spai_pcg_adjoint_device(int64_t n, int64_t a_nnz, const double* a_values, const int64_t* a_indices,
                                const int64_t* a_offsets, int64_t m_nnz, const double* m_values,
                                const int64_t* m_indices, const int64_t* m_offsets, const double* x,
                                const double* grad_x, PcgParams params, double* grad_b, double* grad_a,
                                double* history, int64_t* status, char* error, int64_t error_capacity);
int64_t spai_residual_adjoint_device(int64_t n, int64_t a_nnz, const int64_t* a_col_offsets,
                                     const int64_t* a_row_indices, const double* a_values, int64_t m_nnz,
                                     const int64_t* m_col_offsets, const int64_t* m_row_indices,
                                     const double* m_values, int64_t device, double* loss, double* grad_m,
                                     double* grad_a, char* error, int64_t error_capacity);

/* ---- Matrix Market files, read and written natively (host) ---- */

/* Reads a Matrix Market matrix file (coordinate or array; real, integer or
 * pattern; general, symmetric or skew-symmetric) into the canonical CSC the
 * reference's loader builds (scripts/common.py:397-402: mmread, tocsc,
 * sum_duplicates, eliminate_zeros, sort_indices): symmetric entries mirrored,
 * duplicates summed in file order, explicit zeros removed, rows ascending.
 * threads <= 0: all hardware threads.  The Result carries rows, cols, nnz,
 * col_offsets, row_indices and values (history empty); free it with
 * free_mem.  On failure only error_message is set. */
struct Result spai_mtx_read(const char* path, int64_t threads);

/* Writes CSC m as "%%MatrixMarket matrix coordinate real general" (or
 * "symmetric" with only the entries on or below the diagonal; the caller
 * vouches for the symmetry), 1-based, values with 17 significant digits so
 * that they read back to the same bits.  Returns 0, or -1 with `error`. */
int64_t spai_mtx_write(const char* path, struct MatrixData m, int64_t symmetric, char* error,
                       int64_t error_capacity);

/* y = A x for CSR A (backward_error.pyx:56-66 `matvec`); returns 0, or -1 with `error`. */
int64_t spai_matvec(int64_t n, const double* values, const int64_t* indices, const int64_t* offsets,
                    const double* x, double* y, int64_t device, char* error, int64_t error_capacity);

/* ---- Sessions: the problem stays resident in HBM across repeated runs ---- */
typedef struct SpaiSession SpaiSession;

/* Validates and uploads A (and M0 / Pr when params.use_initial_m /
 * use_preconditioner), builds the row-compressed copy of A, the column norms
 * and the preconditioner.  Returns NULL and fills `error` on failure. */
SpaiSession* spai_session_create(int64_t method, struct MatrixData A, struct MatrixData M0, struct MatrixData Pr,
                                 struct MethodParams params, const SpaiExtParams* ext, char* error,
                                 int64_t error_capacity);
/* The same with the problem already in DEVICE memory (for example the arrays
 * of a torch sparse CSC tensor on the GPU), with no host round trip: A (and
 * M0 when params.use_initial_m) as canonical CSC -- int64 col_offsets (n + 1)
 * running from 0 to nnz, int64 row_indices strictly increasing in every
 * column, FP64 values -- on the session's device, checked there.  Pr is
 * diag(A)^-1 (params.use_preconditioner must be 0).  The caller's arrays are
 * read during the call only; finish writing them before calling. */
SpaiSession* spai_session_create_device(int64_t method, int64_t n, int64_t a_nnz, const int64_t* a_col_offsets,
                                        const int64_t* a_row_indices, const double* a_values, int64_t m0_nnz,
                                        const int64_t* m0_col_offsets, const int64_t* m0_row_indices,
                                        const double* m0_values, struct MethodParams params,
                                        const SpaiExtParams* ext, char* error, int64_t error_capacity);
/* M of the last run into DEVICE arrays on the session's device: col_offsets
 * (n + 1 int64), row_indices and values (capacity >= nnz(M) int64 / double).
 * Returns nnz(M) (the copies are complete), or -1 with `error`. */
int64_t spai_session_result_device(SpaiSession* session, int64_t* col_offsets, int64_t* row_indices, double* values,
                                   int64_t capacity, char* error, int64_t error_capacity);
/* Runs the method from M0 on the resident problem; M stays on the device.
 * Returns 0 (sets *iterations, *converged, *nnz_m), or -1 with `error`. */
int64_t spai_session_run(SpaiSession* session, int64_t* iterations, int64_t* converged, int64_t* nnz_m,
                         char* error, int64_t error_capacity);
/* Copies up to `capacity` history rows of the last run; returns the row count. */
int64_t spai_session_history(SpaiSession* session, struct SingleIterationData* out, int64_t capacity);
/* M of the last run as a Result (free with free_mem). */
struct Result spai_session_result(SpaiSession* session);
/* Uploads the right-hand side b (n doubles) used by spai_session_pcg. */
int64_t spai_session_set_rhs(SpaiSession* session, const double* b, char* error, int64_t error_capacity);
/* PCG on the resident A, the M of the last run (row-compressed on the device,
 * FP32 when params.m_precision == 1) and the resident b.  Same outputs as
 * spai_pcg (x_out may be NULL). */
int64_t spai_session_pcg(SpaiSession* session, PcgParams params, double* history, int64_t* status, double* x_out,
                         char* error, int64_t error_capacity);
void spai_session_destroy(SpaiSession* session);

/* The CUDA stream (cudaStream_t) every kernel of the session runs on, for
 * callers that time the session with their own CUDA events. */
void* spai_session_stream(SpaiSession* session);

/* Fault injection for tests: after `after` more growing device
 * reservations, the next one fails as if the device were out of memory (once;
 * -1 disarms).  The failing call reports the error through its usual error
 * path and releases what it held; the library stays usable. */
void spai_inject_allocation_failure(int64_t after);

/* The device's minimum-norm 2x2 least-squares solve (the per-column step of
 * Inner-Outer LOMR, reference src/common/sparse_operations.cpp:58-73) on
 * `count` systems: gram holds 4 doubles per system (row-major), rhs 2, out
 * receives 2 (host arrays).  Exposes the device arithmetic to tests of the
 * singular and non-finite branches.  Returns 0, or -1 with `error`. */
int64_t spai_solve_2x2_device(int64_t count, const double* gram, const double* rhs, double* out, char* error,
                              int64_t error_capacity);

/* Number of kernels this library has launched since load (diagnostics). */
int64_t spai_kernel_launches(void);

/* Global MR with per-column top-k, a diagonal Pr and a stencil-like A runs
 * its iterations as one CUDA graph of fused kernels (no host round trip per
 * iteration).  enabled = 0 routes every run through the unfused kernels
 * instead; both give the same bits (process-wide, default 1).  No
 * counterpart in the reference. */
void spai_set_fused_mr(int64_t enabled);

/* Opt-in per-kernel-class accounting with CUDA events: enable (1) / disable (0),
 * reset, and read the totals of one class ("spgemm_numeric", "spgemm_symbolic",
 * "union", "transpose", "filter", "pcg_spmv"): elapsed ms, launches and the
 * algorithmic bytes those launches must move.  Returns 1 if the class was seen. */
void spai_profile_enable(int64_t on);
void spai_profile_reset(void);
int64_t spai_profile_read(const char* name, double* ms, int64_t* launches, double* bytes);

#ifdef __cplusplus
}
#endif

#endif /* SPAI_B200_H_ */
