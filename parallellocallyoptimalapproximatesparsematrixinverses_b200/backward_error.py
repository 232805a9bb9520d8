"""PCG evaluator on the device, mirroring the reference's
methods_cython/backward_error.pyx (`pcg`, `matvec`, `parallel_threads`,
backward_error.pyx:45-144) on top of libspai_b200.so.

`pcg` keeps the reference's signature and return value ((history, status));
`threads` is validated as in the reference and otherwise unused because the
work runs on the GPU.  Extra keyword arguments: refresh_period (periodic
true-residual replacement), m_precision ("fp64" | "mixed": M stored in FP32)
and device.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_PF64 = ctypes.POINTER(ctypes.c_double)
_PI64 = ctypes.POINTER(ctypes.c_int64)
M_PRECISIONS = {"fp64": 0, "mixed": 1}


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def parallel_threads(n, requested):
    """backward_error.pyx:45-53: the worker count a PCG call would use."""
    if n <= 0 or requested <= 0:
        raise ValueError("n and requested must be positive")
    return min(n, requested)


def matvec(values, indices, offsets, x, threads, device=-1):
    """y = A x for CSR A (backward_error.pyx:56-66)."""
    offsets = _i64(offsets)
    x = _f64(x)
    if threads <= 0 or offsets.shape[0] != x.shape[0] + 1:
        raise ValueError("Invalid matrix-vector dimensions or thread count")
    values = _f64(values)
    indices = _i64(indices)
    y = np.empty(x.shape[0], dtype=np.float64)
    err = _lib.error_buffer()
    rc = _lib.load().spai_matvec(x.shape[0], values.ctypes.data_as(_PF64), indices.ctypes.data_as(_PI64),
                                 offsets.ctypes.data_as(_PI64), x.ctypes.data_as(_PF64), y.ctypes.data_as(_PF64),
                                 device, err, len(err))
    if rc != 0:
        raise RuntimeError(err.value.decode("utf-8", "replace"))
    return y


def pcg(a_values, a_indices, a_offsets, m_values, m_indices, m_offsets, b, max_iterations, threads, tolerance,
        refresh_period=0, m_precision="fp64", device=-1, return_x=False, symmetric_part=False):
    """PCG with x0 = 0 (backward_error.pyx:69-144); returns (history, status)."""
    b = _f64(b)
    n = b.shape[0]
    if n <= 0 or max_iterations <= 0 or threads <= 0:
        raise ValueError("n, max_iterations and threads must be positive")
    av, ai, ao = _f64(a_values), _i64(a_indices), _i64(a_offsets)
    mv, mi, mo = _f64(m_values), _i64(m_indices), _i64(m_offsets)
    params = _lib.PcgParams(int(max_iterations), float(tolerance), int(refresh_period), M_PRECISIONS[m_precision],
                            int(device), 1 if symmetric_part else 0)
    history = np.zeros(int(max_iterations), dtype=np.float64)
    status = ctypes.c_int64(0)
    x = np.zeros(n, dtype=np.float64) if return_x else None
    err = _lib.error_buffer()
    count = _lib.load().spai_pcg(n, av.ctypes.data_as(_PF64), ai.ctypes.data_as(_PI64), ao.ctypes.data_as(_PI64),
                                 mv.ctypes.data_as(_PF64), mi.ctypes.data_as(_PI64), mo.ctypes.data_as(_PI64),
                                 b.ctypes.data_as(_PF64), params, history.ctypes.data_as(_PF64),
                                 ctypes.byref(status), x.ctypes.data_as(_PF64) if x is not None else None,
                                 err, len(err))
    if count < 0:
        raise RuntimeError(err.value.decode("utf-8", "replace"))
    out = (history[:count].copy(), int(status.value))
    return out + (x,) if return_x else out
