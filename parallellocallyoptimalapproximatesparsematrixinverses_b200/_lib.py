"""ctypes binding of libspai_b200.so (the C ABI in include/methods_c_api.h and
include/spai_b200.h).

The library is built in-tree by build.py.  Loading fails loudly when the
shared object is missing and cannot be built, and every compute call raises
when no CUDA device is present: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_PATH = PACKAGE_DIR / "libspai_b200.so"

_i64 = ctypes.c_int64
_f64 = ctypes.c_double
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pf64 = ctypes.POINTER(ctypes.c_double)


class MatrixData(ctypes.Structure):
    """include/methods_c_api.h MatrixData (reference include/methods_c_api.h:7-14)."""
    _fields_ = [("rows", _i64), ("cols", _i64), ("nnz", _i64),
                ("col_offsets", _pi64), ("row_indices", _pi64), ("values", _pf64)]


class MethodParams(ctypes.Structure):
    """Reference include/methods_c_api.h:16-25."""
    _fields_ = [("max_iterations", _i64), ("tolerance", _f64), ("max_density", _f64),
                ("enable_dropping", _i64), ("num_threads", _i64), ("use_initial_m", _i64),
                ("use_preconditioner", _i64), ("inner_iterations", _i64)]


class SingleIterationData(ctypes.Structure):
    """Reference include/methods_c_api.h:27-32."""
    _fields_ = [("iteration", _i64), ("residual_norm", _f64), ("density_m", _f64),
                ("density_direction", _f64)]


class Result(ctypes.Structure):
    """Reference include/methods_c_api.h:34-46."""
    _fields_ = [("rows", _i64), ("cols", _i64), ("nnz", _i64), ("iterations", _i64),
                ("converged", _i64), ("history_size", _i64), ("col_offsets", _pi64),
                ("row_indices", _pi64), ("values", _pf64),
                ("history", ctypes.POINTER(SingleIterationData)), ("error_message", ctypes.c_char_p)]


class SpaiExtParams(ctypes.Structure):
    """include/spai_b200.h SpaiExtParams."""
    _fields_ = [("precision", _i64), ("topk_per_column", _i64), ("device", _i64), ("summation_order", _i64)]


class PcgParams(ctypes.Structure):
    """include/spai_b200.h PcgParams."""
    _fields_ = [("max_iterations", _i64), ("tolerance", _f64), ("refresh_period", _i64),
                ("m_precision", _i64), ("device", _i64), ("symmetric_part", _i64)]


METHOD_IDS = {
    ("global_spai", "cg"): 0,
    ("global_spai", "mr"): 1,
    ("global_spai", "lomr"): 2,
    ("inner_outer", "mr"): 3,
    ("inner_outer", "lomr"): 4,
}

# entry point name -> method id, the five reference symbols (methods_c_api.h:48-56)
REFERENCE_ENTRY_POINTS = {
    "spai_global_cg": 0,
    "spai_global_mr": 1,
    "spai_global_lomr": 2,
    "inner_outer_mr": 3,
    "inner_outer_lomr": 4,
}

# every symbol declared in include/*.h
EXPORTED_SYMBOLS = (
    "spai_global_cg", "spai_global_mr", "spai_global_lomr", "inner_outer_mr", "inner_outer_lomr", "free_mem",
    "spai_run_ex", "spai_pcg", "spai_matvec", "spai_session_create", "spai_session_run", "spai_session_history",
    "spai_session_result", "spai_session_set_rhs", "spai_session_pcg", "spai_session_destroy",
    "spai_kernel_launches", "spai_session_stream", "spai_profile_enable", "spai_profile_reset",
    "spai_profile_read", "spai_pcg_device_noalloc", "spai_residual_adjoint", "spai_pcg_adjoint",
    "spai_pcg_device", "spai_pcg_adjoint_device", "spai_residual_adjoint_device",
    "spai_mr_batched", "spai_mtx_read", "spai_mtx_write", "spai_free_int64_array", "spai_free_double_array",
    "spai_session_create_device", "spai_session_result_device", "spai_inject_allocation_failure",
    "spai_set_fused_mr", "spai_solve_2x2_device",
)

_lib = None
_lock = threading.Lock()


def _declare(lib) -> None:
    method_args = [MatrixData, MatrixData, MatrixData, MethodParams]
    for name in REFERENCE_ENTRY_POINTS:
        fn = getattr(lib, name)
        fn.restype = Result
        fn.argtypes = method_args
    lib.free_mem.restype = None
    lib.free_mem.argtypes = [ctypes.POINTER(Result)]
    lib.spai_run_ex.restype = Result
    lib.spai_run_ex.argtypes = [_i64, MatrixData, MatrixData, MatrixData, MethodParams, ctypes.POINTER(SpaiExtParams)]
    lib.spai_pcg.restype = _i64
    lib.spai_pcg.argtypes = [_i64, _pf64, _pi64, _pi64, _pf64, _pi64, _pi64, _pf64, PcgParams, _pf64, _pi64, _pf64,
                             ctypes.c_char_p, _i64]
    lib.spai_matvec.restype = _i64
    lib.spai_matvec.argtypes = [_i64, _pf64, _pi64, _pi64, _pf64, _pf64, _i64, ctypes.c_char_p, _i64]
    lib.spai_session_create.restype = ctypes.c_void_p
    lib.spai_session_create.argtypes = [_i64, MatrixData, MatrixData, MatrixData, MethodParams,
                                        ctypes.POINTER(SpaiExtParams), ctypes.c_char_p, _i64]
    lib.spai_session_run.restype = _i64
    lib.spai_session_run.argtypes = [ctypes.c_void_p, _pi64, _pi64, _pi64, ctypes.c_char_p, _i64]
    lib.spai_session_history.restype = _i64
    lib.spai_session_history.argtypes = [ctypes.c_void_p, ctypes.POINTER(SingleIterationData), _i64]
    lib.spai_session_result.restype = Result
    lib.spai_session_result.argtypes = [ctypes.c_void_p]
    lib.spai_session_set_rhs.restype = _i64
    lib.spai_session_set_rhs.argtypes = [ctypes.c_void_p, _pf64, ctypes.c_char_p, _i64]
    lib.spai_session_pcg.restype = _i64
    lib.spai_session_pcg.argtypes = [ctypes.c_void_p, PcgParams, _pf64, _pi64, _pf64, ctypes.c_char_p, _i64]
    lib.spai_session_destroy.restype = None
    lib.spai_session_destroy.argtypes = [ctypes.c_void_p]
    lib.spai_kernel_launches.restype = _i64
    lib.spai_kernel_launches.argtypes = []
    lib.spai_session_stream.restype = ctypes.c_void_p
    lib.spai_session_stream.argtypes = [ctypes.c_void_p]
    lib.spai_profile_enable.restype = None
    lib.spai_profile_enable.argtypes = [_i64]
    lib.spai_profile_reset.restype = None
    lib.spai_profile_reset.argtypes = []
    lib.spai_profile_read.restype = _i64
    lib.spai_profile_read.argtypes = [ctypes.c_char_p, _pf64, _pi64, _pf64]
    # device pointers are passed as integers (e.g. torch.Tensor.data_ptr())
    lib.spai_pcg_device_noalloc.restype = _i64
    lib.spai_pcg_device_noalloc.argtypes = [_i64, _i64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i64,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, _i64, _f64, _i64, ctypes.c_void_p, _pf64, _pi64,
                                            ctypes.c_char_p, _i64]
    lib.spai_inject_allocation_failure.restype = None
    lib.spai_inject_allocation_failure.argtypes = [_i64]
    lib.spai_set_fused_mr.restype = None
    lib.spai_set_fused_mr.argtypes = [_i64]
    lib.spai_solve_2x2_device.restype = _i64
    lib.spai_solve_2x2_device.argtypes = [_i64, _pf64, _pf64, _pf64, ctypes.c_char_p, _i64]
    lib.spai_session_create_device.restype = ctypes.c_void_p
    lib.spai_session_create_device.argtypes = [_i64, _i64, _i64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               _i64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, MethodParams,
                                               ctypes.POINTER(SpaiExtParams), ctypes.c_char_p, _i64]
    lib.spai_session_result_device.restype = _i64
    lib.spai_session_result_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               _i64, ctypes.c_char_p, _i64]
    lib.spai_free_int64_array.restype = None
    lib.spai_free_int64_array.argtypes = [ctypes.c_void_p]
    lib.spai_free_double_array.restype = None
    lib.spai_free_double_array.argtypes = [ctypes.c_void_p]
    lib.spai_mtx_read.restype = Result
    lib.spai_mtx_read.argtypes = [ctypes.c_char_p, _i64]
    lib.spai_mtx_write.restype = _i64
    lib.spai_mtx_write.argtypes = [ctypes.c_char_p, MatrixData, _i64, ctypes.c_char_p, _i64]
    lib.spai_mr_batched.restype = _i64
    lib.spai_mr_batched.argtypes = [_i64, ctypes.POINTER(MatrixData), ctypes.POINTER(MatrixData), MethodParams,
                                    ctypes.POINTER(SpaiExtParams), ctypes.POINTER(Result), ctypes.c_char_p, _i64]
    lib.spai_residual_adjoint.restype = _i64
    lib.spai_residual_adjoint.argtypes = [MatrixData, MatrixData, _i64, _pf64, _pf64, _pf64, ctypes.c_char_p, _i64]
    _vp = ctypes.c_void_p
    lib.spai_pcg_device.restype = _i64
    lib.spai_pcg_device.argtypes = [_i64, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, PcgParams, _pf64,
                                    ctypes.POINTER(_i64), _vp, ctypes.c_char_p, _i64]
    lib.spai_pcg_adjoint_device.restype = _i64
    lib.spai_pcg_adjoint_device.argtypes = [_i64, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, PcgParams, _vp,
                                            _vp, _pf64, ctypes.POINTER(_i64), ctypes.c_char_p, _i64]
    lib.spai_residual_adjoint_device.restype = _i64
    lib.spai_residual_adjoint_device.argtypes = [_i64, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _pf64, _vp,
                                                 _vp, ctypes.c_char_p, _i64]
    lib.spai_pcg_adjoint.restype = _i64
    lib.spai_pcg_adjoint.argtypes = [_i64, _pf64, _pi64, _pi64, _pf64, _pi64, _pi64, _pf64, _pf64, PcgParams, _pf64,
                                     _pf64, _pf64, _pi64, ctypes.c_char_p, _i64]


def load():
    """Load (building first if needed) libspai_b200.so."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                from . import build as _build
                _build.build()
            lib = ctypes.CDLL(str(LIB_PATH))
            _declare(lib)
            _lib = lib
    return _lib


def error_buffer(size: int = 1024):
    return ctypes.create_string_buffer(size)
