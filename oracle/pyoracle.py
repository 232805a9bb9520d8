"""TEST INFRASTRUCTURE ONLY: ctypes loader for the CPU oracle (libspai_oracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module.  It exposes the oracle's SPAI methods with the same Python surface as
the reference's methods_cython.methods (reference methods_cython/methods.pyx:74-179)
plus the oracle options (summation order, batch count, per-column top-k), and
the oracle PCG (reference methods_cython/backward_error.pyx:69-144).
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
from scipy import sparse

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libspai_oracle.so"

METHOD_IDS = {
    ("global_spai", "cg"): 0,
    ("global_spai", "mr"): 1,
    ("global_spai", "lomr"): 2,
    ("inner_outer", "mr"): 3,
    ("inner_outer", "lomr"): 4,
}

ORDER_REFERENCE = 0
ORDER_DEVICE = 1

_i64 = ctypes.c_int64
_f64 = ctypes.c_double
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pf64 = ctypes.POINTER(ctypes.c_double)


class MatrixData(ctypes.Structure):
    _fields_ = [("rows", _i64), ("cols", _i64), ("nnz", _i64),
                ("col_offsets", _pi64), ("row_indices", _pi64), ("values", _pf64)]


class MethodParams(ctypes.Structure):
    _fields_ = [("max_iterations", _i64), ("tolerance", _f64), ("max_density", _f64),
                ("enable_dropping", _i64), ("num_threads", _i64), ("use_initial_m", _i64),
                ("use_preconditioner", _i64), ("inner_iterations", _i64)]


class SingleIterationData(ctypes.Structure):
    _fields_ = [("iteration", _i64), ("residual_norm", _f64), ("density_m", _f64),
                ("density_direction", _f64)]


class Result(ctypes.Structure):
    _fields_ = [("rows", _i64), ("cols", _i64), ("nnz", _i64), ("iterations", _i64),
                ("converged", _i64), ("history_size", _i64), ("col_offsets", _pi64),
                ("row_indices", _pi64), ("values", _pf64),
                ("history", ctypes.POINTER(SingleIterationData)), ("error_message", ctypes.c_char_p)]


class OracleOptions(ctypes.Structure):
    _fields_ = [("order", _i64), ("batch_count", _i64), ("omp_threads", _i64),
                ("topk_per_column", _i64)]


HISTORY_DTYPE = np.dtype([("iteration", np.int64), ("residual_norm", np.float64),
                          ("density_m", np.float64), ("density_direction", np.float64)])

_lib = None


def build() -> None:
    """Compile the oracle library (needs g++ with OpenMP)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.oracle_run.restype = Result
        _lib.oracle_run.argtypes = [_i64, MatrixData, MatrixData, MatrixData, MethodParams, OracleOptions]
        _lib.oracle_free.restype = None
        _lib.oracle_free.argtypes = [ctypes.POINTER(Result)]
        _lib.oracle_pcg.restype = _i64
        _lib.oracle_pcg.argtypes = [_i64, _pf64, _pi64, _pi64, _pf64, _pi64, _pi64, _pf64, _i64, _f64,
                                    _i64, _i64, _pf64, _pi64, _pf64]
        _lib.oracle_tree_sum.restype = _f64
        _lib.oracle_tree_sum.argtypes = [_pf64, _i64]
        _lib.oracle_solve_2x2.restype = None
        _lib.oracle_solve_2x2.argtypes = [_pf64, _pf64, _pf64]
    return _lib


class OutputResult:
    """Same fields as the reference's methods_cython OutputResult (methods.pyx:61-67)."""

    def __init__(self, M, iterations, converged, history):
        self.M = M
        self.iterations = iterations
        self.converged = converged
        self.history = history
        self.residual_norms = history["residual_norm"]


def as_csc(matrix, shape=None):
    """scipy -> canonical CSC with int64 indices (reference methods.pyx:74-87)."""
    if matrix is None:
        return sparse.csc_matrix((0, 0), dtype=np.float64)
    csc = sparse.csc_matrix(matrix, dtype=np.float64, copy=True)
    if shape is not None and csc.shape != tuple(shape):
        raise ValueError("matrix shape does not match A")
    csc.sum_duplicates()
    csc.sort_indices()
    csc.indptr = np.ascontiguousarray(csc.indptr, dtype=np.int64)
    csc.indices = np.ascontiguousarray(csc.indices, dtype=np.int64)
    csc.data = np.ascontiguousarray(csc.data, dtype=np.float64)
    return csc


def _matrix_data(csc) -> MatrixData:
    return MatrixData(csc.shape[0], csc.shape[1], csc.nnz,
                      csc.indptr.ctypes.data_as(_pi64), csc.indices.ctypes.data_as(_pi64),
                      csc.data.ctypes.data_as(_pf64))


def result_to_python(res: Result, free) -> OutputResult:
    try:
        if res.error_message:
            raise RuntimeError(res.error_message.decode("utf-8", "replace"))
        indptr = np.ctypeslib.as_array(res.col_offsets, shape=(res.cols + 1,)).copy()
        if res.nnz:
            indices = np.ctypeslib.as_array(res.row_indices, shape=(res.nnz,)).copy()
            values = np.ctypeslib.as_array(res.values, shape=(res.nnz,)).copy()
        else:
            indices = np.empty(0, dtype=np.int64)
            values = np.empty(0, dtype=np.float64)
        M = sparse.csc_matrix((values, indices, indptr), shape=(res.rows, res.cols))
        history = np.empty(res.history_size, dtype=HISTORY_DTYPE)
        for i in range(res.history_size):
            h = res.history[i]
            history[i] = (h.iteration, h.residual_norm, h.density_m, h.density_direction)
        return OutputResult(M, res.iterations, bool(res.converged), history)
    finally:
        free(ctypes.byref(res))


def run(family: str, method: str, A, M0=None, Pr=None, max_iterations=100, tolerance=1e-9,
        max_density=0.03, enable_dropping=True, num_threads=1, inner_iterations=2,
        order=ORDER_REFERENCE, batch_count=0, omp_threads=0, topk_per_column=0) -> OutputResult:
    """Run one oracle method; arguments follow methods_cython (methods.pyx:147-179)."""
    L = lib()
    A_csc = as_csc(A)
    M0_csc = as_csc(M0, A_csc.shape) if M0 is not None else as_csc(None)
    Pr_csc = as_csc(Pr, A_csc.shape) if Pr is not None else as_csc(None)
    params = MethodParams(max_iterations, tolerance, max_density, 1 if enable_dropping else 0, num_threads,
                          1 if M0 is not None else 0, 1 if Pr is not None else 0, inner_iterations)
    opts = OracleOptions(order, batch_count, omp_threads, topk_per_column)
    res = L.oracle_run(METHOD_IDS[(family, method)], _matrix_data(A_csc), _matrix_data(M0_csc),
                       _matrix_data(Pr_csc), params, opts)
    return result_to_python(res, L.oracle_free)


def pcg(A, M, b, max_iterations, tolerance, order=ORDER_REFERENCE, refresh_period=0, return_x=False):
    """Oracle PCG on CSR A and M; returns (history, status[, x])."""
    L = lib()
    A = sparse.csr_matrix(A, dtype=np.float64)
    M = sparse.csr_matrix(M, dtype=np.float64)
    n = A.shape[0]
    av, ai, ao = (np.ascontiguousarray(A.data, np.float64), np.ascontiguousarray(A.indices, np.int64),
                  np.ascontiguousarray(A.indptr, np.int64))
    mv, mi, mo = (np.ascontiguousarray(M.data, np.float64), np.ascontiguousarray(M.indices, np.int64),
                  np.ascontiguousarray(M.indptr, np.int64))
    b = np.ascontiguousarray(b, np.float64)
    history = np.zeros(max_iterations, np.float64)
    x = np.zeros(n, np.float64)
    status = ctypes.c_int64(0)
    count = L.oracle_pcg(n, av.ctypes.data_as(_pf64), ai.ctypes.data_as(_pi64), ao.ctypes.data_as(_pi64),
                         mv.ctypes.data_as(_pf64), mi.ctypes.data_as(_pi64), mo.ctypes.data_as(_pi64),
                         b.ctypes.data_as(_pf64), max_iterations, tolerance, order, refresh_period,
                         history.ctypes.data_as(_pf64), ctypes.byref(status), x.ctypes.data_as(_pf64))
    out = (history[:count].copy(), int(status.value))
    return out + (x,) if return_x else out


def tree_sum(values) -> float:
    v = np.ascontiguousarray(values, np.float64)
    return float(lib().oracle_tree_sum(v.ctypes.data_as(_pf64), v.size))


def solve_2x2(matrix, rhs):
    m = np.ascontiguousarray(np.asarray(matrix, np.float64).reshape(4))
    r = np.ascontiguousarray(np.asarray(rhs, np.float64).reshape(2))
    out = np.zeros(2, np.float64)
    lib().oracle_solve_2x2(m.ctypes.data_as(_pf64), r.ctypes.data_as(_pf64), out.ctypes.data_as(_pf64))
    return out


def reference_pcg_module():
    """The reference's own backward_error module compiled into oracle/_ref (or None)."""
    import importlib.util
    ref_dir = HERE / "_ref"
    for path in sorted(ref_dir.glob("backward_error*.so")):
        spec = importlib.util.spec_from_file_location("backward_error", path)
        module = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(module)
        return module
    return None
