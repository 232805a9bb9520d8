"""Python surface of the SPAI methods, mirroring the reference's
methods_cython/methods.pyx (GlobalSpaiMethods / InnerOuterMethods,
methods.pyx:182-258) on top of libspai_b200.so.

    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import global_spai
    result = global_spai.mr(A, M0=M0, Pr=Pr, max_iterations=20, max_density=10 / n)
    result.M, result.iterations, result.converged, result.history

Same arguments, defaults, conversions (scipy -> canonical int64 CSC, methods.pyx:74-98)
and error behaviour (RuntimeError with the library's message, methods.pyx:128-130)
as the reference.  Extra keyword arguments select the device-only forms:
precision ("fp64" | "mixed"), topk_per_column (0 = the reference's global budget),
device (CUDA ordinal, -1 = current) and summation ("device" | "reference": the
reference's num_threads column batches and summation order, which reproduces
its recorded results bit for bit in FP64).  Left unset, summation follows the
precision: an FP64 run with the reference's global budget (no top-k) uses the
reference's order, so a call with only the reference's arguments returns the
reference's bits; the extension forms (mixed precision, per-column top-k) use
the device order.
"""
from __future__ import annotations

import ctypes
from concurrent.futures import ThreadPoolExecutor

import numpy as np
from scipy import sparse

from . import _lib

HISTORY_DTYPE = np.dtype([
    ("iteration", np.int64),
    ("residual_norm", np.float64),
    ("density_m", np.float64),
    ("density_direction", np.float64),
])

PRECISIONS = {"fp64": 0, "mixed": 1}
# "device": per-column sums and the fixed tree; "reference": the reference's
# num_threads column batches, summed in its order (its recorded results, bit for bit)
SUMMATIONS = {"device": 0, "reference": 1}


class OutputResult:
    """Reference methods_cython/methods.pyx:61-67."""

    def __init__(self, M, iterations, converged, history):
        self.M = M
        self.iterations = iterations
        self.converged = converged
        self.history = history
        self.residual_norms = history["residual_norm"]


def _empty_csc():
    return sparse.csc_matrix((0, 0), dtype=np.float64)


def as_csc(matrix, shape=None):
    """scipy matrix -> canonical CSC with int64 indices (methods.pyx:74-87)."""
    if matrix is None:
        return _empty_csc()
    csc = sparse.csc_matrix(matrix, dtype=np.float64, copy=False)
    if shape is not None and csc.shape != tuple(shape):
        raise ValueError("matrix shape does not match A")
    csc.sum_duplicates()
    csc.sort_indices()
    csc.indptr = np.ascontiguousarray(csc.indptr, dtype=np.int64)
    csc.indices = np.ascontiguousarray(csc.indices, dtype=np.int64)
    csc.data = np.ascontiguousarray(csc.data, dtype=np.float64)
    return csc


def matrix_data(csc) -> _lib.MatrixData:
    """Borrowed pointers into a canonical CSC (methods.pyx:90-98)."""
    return _lib.MatrixData(
        csc.shape[0], csc.shape[1], csc.nnz,
        csc.indptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
        csc.indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
        csc.data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
    )


def history_array(rows, count) -> np.ndarray:
    history = np.empty(count, dtype=HISTORY_DTYPE)
    for i in range(count):
        h = rows[i]
        history[i] = (h.iteration, h.residual_norm, h.density_m, h.density_direction)
    return history


class _LibraryArray:
    """Owner of one array of a Result: numpy views of it keep this object
    alive, and the last one to go releases the array through the library."""

    def __init__(self, address, count, typestr, release):
        self.address = address
        self._release = release
        self.__array_interface__ = {"data": (address, False), "shape": (count,), "typestr": typestr, "version": 3}

    def __del__(self):
        try:
            self._release(self.address)
        except Exception:  # interpreter shutdown: the process frees the memory
            pass


def adopt_matrix(result: _lib.Result) -> sparse.csc_matrix:
    """M of a successful Result as a scipy CSC matrix whose arrays are the
    library's own (no copy); clears the Result's matrix fields, so that
    free_mem releases only the rest."""
    lib = _lib.load()
    arrays = []
    for field, typestr, count, release in (("col_offsets", "<i8", result.cols + 1, lib.spai_free_int64_array),
                                           ("row_indices", "<i8", result.nnz, lib.spai_free_int64_array),
                                           ("values", "<f8", result.nnz, lib.spai_free_double_array)):
        address = ctypes.cast(getattr(result, field), ctypes.c_void_p).value
        setattr(result, field, None)
        arrays.append(np.asarray(_LibraryArray(address, count, typestr, release)))
    indptr, indices, values = arrays
    # assigned, not passed to the constructor: scipy would scan the indices and
    # copy them down to int32; the library's columns are sorted and duplicate-free
    m = sparse.csc_matrix((result.rows, result.cols), dtype=np.float64)
    m.data, m.indices, m.indptr = values, indices, indptr
    m.has_canonical_format = True
    return m


def result_to_python(result: _lib.Result) -> OutputResult:
    """Turns a Result into numpy/scipy and always frees it (methods.pyx:119-144);
    M keeps the library's arrays instead of copying them."""
    lib = _lib.load()
    try:
        if result.error_message:
            raise RuntimeError(result.error_message.decode("utf-8", "replace"))
        M = adopt_matrix(result)
        history = history_array(result.history, result.history_size)
        return OutputResult(M, result.iterations, bool(result.converged), history)
    finally:
        lib.free_mem(ctypes.byref(result))


def method_params(A_csc, M0, Pr, max_iterations, tolerance, max_density, enable_dropping, num_threads,
                  inner_iterations) -> _lib.MethodParams:
    return _lib.MethodParams(max_iterations, tolerance, max_density, 1 if enable_dropping else 0, num_threads,
                             1 if M0 is not None else 0, 1 if Pr is not None else 0, inner_iterations)


def ext_params(precision="fp64", topk_per_column=0, device=-1, summation="device") -> _lib.SpaiExtParams:
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    if summation not in SUMMATIONS:
        raise ValueError(f"summation must be one of {sorted(SUMMATIONS)}")
    return _lib.SpaiExtParams(PRECISIONS[precision], int(topk_per_column), int(device), SUMMATIONS[summation])


def default_summation(precision="fp64", topk_per_column=0) -> str:
    """The summation order of a run that does not name one: the reference's
    for its own form (FP64, global budget), the device order otherwise."""
    return "reference" if precision == "fp64" and not topk_per_column else "device"


def _call_method(family, name, A, M0, Pr, max_iterations, tolerance, max_density, enable_dropping, num_threads,
                 inner_iterations=2, precision="fp64", topk_per_column=0, device=-1,
                 summation=None) -> OutputResult:
    """methods.pyx:147-179 plus the extension knobs."""
    if summation is None:
        summation = default_summation(precision, topk_per_column)
    lib = _lib.load()
    A_csc = as_csc(A)
    M0_csc = as_csc(M0, A_csc.shape) if M0 is not None else _empty_csc()
    Pr_csc = as_csc(Pr, A_csc.shape) if Pr is not None else _empty_csc()
    params = method_params(A_csc, M0, Pr, max_iterations, tolerance, max_density, enable_dropping, num_threads,
                           inner_iterations)
    method_id = _lib.METHOD_IDS[(family, name)]
    if precision == "fp64" and not topk_per_column and device == -1 and summation == "reference":
        # the reference's own entry points (methods_c_api.h:48-56), which run in its summation order
        entry = {0: lib.spai_global_cg, 1: lib.spai_global_mr, 2: lib.spai_global_lomr,
                 3: lib.inner_outer_mr, 4: lib.inner_outer_lomr}[method_id]
        result = entry(matrix_data(A_csc), matrix_data(M0_csc), matrix_data(Pr_csc), params)
    else:
        ext = ext_params(precision, topk_per_column, device, summation)
        result = lib.spai_run_ex(method_id, matrix_data(A_csc), matrix_data(M0_csc), matrix_data(Pr_csc), params,
                                 ctypes.byref(ext))
    return result_to_python(result)


class GlobalSpaiMethods:
    """Reference methods.pyx:182-222."""
    available_methods = ("cg", "mr", "lomr")

    def cg(self, A, M0=None, Pr=None, max_iterations=100, tolerance=1e-9, max_density=0.03, enable_dropping=True,
           num_threads=1, **ext):
        return _call_method("global_spai", "cg", A, M0, Pr, max_iterations, tolerance, max_density,
                            enable_dropping, num_threads, **ext)

    def mr(self, A, M0=None, Pr=None, max_iterations=100, tolerance=1e-9, max_density=0.03, enable_dropping=True,
           num_threads=1, **ext):
        return _call_method("global_spai", "mr", A, M0, Pr, max_iterations, tolerance, max_density,
                            enable_dropping, num_threads, **ext)

    def lomr(self, A, M0=None, Pr=None, max_iterations=100, tolerance=1e-9, max_density=0.03, enable_dropping=True,
             num_threads=1, **ext):
        return _call_method("global_spai", "lomr", A, M0, Pr, max_iterations, tolerance, max_density,
                            enable_dropping, num_threads, **ext)

    def mr_batched(self, As, M0s=None, max_iterations=100, tolerance=1e-9, max_density=0.03, enable_dropping=True,
                   num_threads=1, topk_per_column=0, precision="fp64", device=-1):
        """`mr` on many independent systems in one batch (libspai_b200.so
        spai_mr_batched): one list entry per system, each what `mr` returns
        for that system alone with Pr = diag(A)^-1.  Dropping, when enabled,
        must be per column (topk_per_column > 0)."""
        lib = _lib.load()
        As = list(As)
        count = len(As)
        if count == 0:
            return []
        if M0s is not None and len(M0s) != count:
            raise ValueError("M0s must have one matrix per system")
        # canonical int64 CSC per system; numpy's copies release the GIL, so large batches convert on threads
        with ThreadPoolExecutor(max_workers=min(8, count)) as pool:
            As = list(pool.map(as_csc, As))
            if M0s is not None:
                M0s = list(pool.map(lambda pair: as_csc(pair[0], pair[1].shape), zip(M0s, As)))
        params = _lib.MethodParams(max_iterations, tolerance, max_density, 1 if enable_dropping else 0, num_threads,
                                   1 if M0s is not None else 0, 0, 2)
        ext = ext_params(precision, topk_per_column, device)
        a_data = (_lib.MatrixData * count)(*[matrix_data(A) for A in As])
        m_data = (_lib.MatrixData * count)(*[matrix_data(M) for M in M0s]) if M0s is not None else None
        results = (_lib.Result * count)()
        err = _lib.error_buffer()
        rc = lib.spai_mr_batched(count, a_data, m_data, params, ctypes.byref(ext), results, err, len(err))
        if rc != 0:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        out = []
        for b in range(count):
            out.append(result_to_python(results[b]))
        return out


class InnerOuterMethods:
    """Reference methods.pyx:225-254."""
    available_methods = ("mr", "lomr")

    def mr(self, A, M0=None, Pr=None, max_iterations=100, tolerance=1e-9, max_density=0.03, enable_dropping=True,
           num_threads=1, inner_iterations=2, **ext):
        return _call_method("inner_outer", "mr", A, M0, Pr, max_iterations, tolerance, max_density,
                            enable_dropping, num_threads, inner_iterations, **ext)

    def lomr(self, A, M0=None, Pr=None, max_iterations=100, tolerance=1e-9, max_density=0.03, enable_dropping=True,
             num_threads=1, inner_iterations=2, **ext):
        return _call_method("inner_outer", "lomr", A, M0, Pr, max_iterations, tolerance, max_density,
                            enable_dropping, num_threads, inner_iterations, **ext)


global_spai = GlobalSpaiMethods()
inner_outer = InnerOuterMethods()


class Session:
    """A problem resident in HBM (include/spai_b200.h sessions): repeated SPAI
    runs and PCG solves without re-uploading A."""

    def __init__(self, family, name, A, M0=None, Pr=None, max_iterations=100, tolerance=1e-9, max_density=0.03,
                 enable_dropping=True, num_threads=1, inner_iterations=2, precision="fp64", topk_per_column=0,
                 device=-1):
        self._lib = _lib.load()
        self._A = as_csc(A)
        self._M0 = as_csc(M0, self._A.shape) if M0 is not None else _empty_csc()
        self._Pr = as_csc(Pr, self._A.shape) if Pr is not None else _empty_csc()
        params = method_params(self._A, M0, Pr, max_iterations, tolerance, max_density, enable_dropping,
                               num_threads, inner_iterations)
        ext = ext_params(precision, topk_per_column, device)
        err = _lib.error_buffer()
        handle = self._lib.spai_session_create(_lib.METHOD_IDS[(family, name)], matrix_data(self._A),
                                               matrix_data(self._M0), matrix_data(self._Pr), params,
                                               ctypes.byref(ext), err, len(err))
        if not handle:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        self._handle = ctypes.c_void_p(handle)
        self.n = self._A.shape[0]
        self._nnz = 0

    @classmethod
    def from_torch(cls, family, name, A, M0=None, max_iterations=100, tolerance=1e-9, max_density=0.03,
                   enable_dropping=True, num_threads=1, inner_iterations=2, precision="fp64", topk_per_column=0,
                   summation="device"):
        """A session on the GPU arrays of torch sparse CSC tensors -- A, and M0
        when given -- with no host round trip (spai_session_create_device):
        float64 values on one CUDA device, rows sorted and unique in every
        column (checked on the device).  Pr is diag(A)^-1."""
        import torch
        tensors = [A] + ([M0] if M0 is not None else [])
        for t in tensors:
            if t.layout != torch.sparse_csc or not t.is_cuda or t.dtype != torch.float64:
                raise ValueError("A and M0 must be float64 torch.sparse_csc tensors on a CUDA device")
            if t.shape[0] != t.shape[1] or t.shape != A.shape or t.device != A.device:
                raise ValueError("A and M0 must be square, of one size and on one device")
        arrays = [(t.ccol_indices().to(torch.int64).contiguous(), t.row_indices().to(torch.int64).contiguous(),
                   t.values().contiguous()) for t in tensors]
        torch.cuda.synchronize(A.device)  # the arrays are complete before the library reads them on its stream
        self = cls.__new__(cls)
        self._lib = _lib.load()
        n = A.shape[0]
        params = _lib.MethodParams(max_iterations, tolerance, max_density, 1 if enable_dropping else 0, num_threads,
                                   1 if M0 is not None else 0, 0, inner_iterations)
        ext = ext_params(precision, topk_per_column, A.device.index, summation)
        a_ptr, a_idx, a_val = arrays[0]
        m_ptr, m_idx, m_val = arrays[1] if M0 is not None else (None, None, None)
        err = _lib.error_buffer()
        handle = self._lib.spai_session_create_device(
            _lib.METHOD_IDS[(family, name)], n, a_val.numel(), a_ptr.data_ptr(), a_idx.data_ptr(), a_val.data_ptr(),
            m_val.numel() if m_val is not None else 0, m_ptr.data_ptr() if m_ptr is not None else None,
            m_idx.data_ptr() if m_idx is not None else None, m_val.data_ptr() if m_val is not None else None,
            params, ctypes.byref(ext), err, len(err))
        if not handle:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        self._handle = ctypes.c_void_p(handle)
        self.n = n
        self._nnz = 0
        self._device = A.device
        return self

    def result_torch(self):
        """M of the last run as a float64 torch.sparse_csc tensor on the
        session's device (spai_session_result_device; no host round trip)."""
        import torch
        device = getattr(self, "_device", None) or torch.device("cuda", torch.cuda.current_device())
        ptr = torch.empty(self.n + 1, dtype=torch.int64, device=device)
        idx = torch.empty(max(self._nnz, 1), dtype=torch.int64, device=device)
        val = torch.empty(max(self._nnz, 1), dtype=torch.float64, device=device)
        err = _lib.error_buffer()
        nnz = self._lib.spai_session_result_device(self._handle, ptr.data_ptr(), idx.data_ptr(), val.data_ptr(),
                                                   idx.numel(), err, len(err))
        if nnz < 0:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        return torch.sparse_csc_tensor(ptr, idx[:nnz], val[:nnz], size=(self.n, self.n))

    def run(self):
        it = ctypes.c_int64(0)
        conv = ctypes.c_int64(0)
        nnz = ctypes.c_int64(0)
        err = _lib.error_buffer()
        if self._lib.spai_session_run(self._handle, ctypes.byref(it), ctypes.byref(conv), ctypes.byref(nnz), err,
                                      len(err)) != 0:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        self._nnz = nnz.value
        self.converged = bool(conv.value)
        return it.value, nnz.value

    def history(self):
        cap = 1 << 16
        rows = (_lib.SingleIterationData * cap)()
        count = self._lib.spai_session_history(self._handle, rows, cap)
        return history_array(rows, min(count, cap))

    def result(self) -> OutputResult:
        return result_to_python(self._lib.spai_session_result(self._handle))

    def set_rhs(self, b):
        self._b = np.ascontiguousarray(b, dtype=np.float64)
        err = _lib.error_buffer()
        if self._lib.spai_session_set_rhs(self._handle, self._b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), err,
                                          len(err)) != 0:
            raise RuntimeError(err.value.decode("utf-8", "replace"))

    def pcg(self, max_iterations, tolerance, refresh_period=0, m_precision="fp64", return_x=False, device=-1,
            symmetric_part=False):
        params = _lib.PcgParams(max_iterations, tolerance, refresh_period, PRECISIONS[m_precision], device,
                                1 if symmetric_part else 0)
        history = np.zeros(max_iterations, dtype=np.float64)
        status = ctypes.c_int64(0)
        x = np.zeros(self.n, dtype=np.float64) if return_x else None
        err = _lib.error_buffer()
        count = self._lib.spai_session_pcg(self._handle, params,
                                           history.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                           ctypes.byref(status),
                                           x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if x is not None else None,
                                           err, len(err))
        if count < 0:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        out = (history[:count].copy(), int(status.value))
        return out + (x,) if return_x else out

    @property
    def stream(self) -> int:
        """cudaStream_t of the session (for CUDA events recorded by the caller)."""
        return int(self._lib.spai_session_stream(self._handle) or 0)

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.spai_session_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
