"""Reverse mode on the device: gradients of the SPAI objective and of the PCG
solve, as functions on scipy matrices and as torch.autograd.Function objects.

The reference has no adjoint.  These differentiate the two quantities it does
compute:

* f(A, M) = ||I - A M||_F^2, the square of the residual norm that every SPAI
  iteration records (methods_common.cpp:112-122).  `residual_adjoint` returns
  f with df/dM on M's pattern and df/dA on A's pattern
  (libspai_b200.so `spai_residual_adjoint`).
* x = A^-1 b by PCG (backward_error.pyx:69-144).  `pcg_adjoint` maps an
  upstream gradient dL/dx to dL/db and dL/dA on A's pattern by one more PCG
  solve with the forward's preconditioner (`spai_pcg_adjoint`; the
  implicit-function adjoint, exact for the solution map A^-1 b).

`residual_objective` and `pcg_solve` wrap both for torch autograd over the
stored values of fixed sparsity patterns.  CUDA tensors stay on their device:
their pointers go to the device forms of the entry points
(`spai_residual_adjoint_device`, `spai_pcg_device`,
`spai_pcg_adjoint_device`), which give the same bits as the host forms, and
only the patterns (when given as numpy arrays), the loss and the solve's
history cross to or from the host.  CPU tensors go through the host forms.
Gradients come back on the device and in the dtype (float64) of the inputs.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
from scipy import sparse

from . import _lib
from .backward_error import M_PRECISIONS, pcg

_PF64 = ctypes.POINTER(ctypes.c_double)
_PI64 = ctypes.POINTER(ctypes.c_int64)


def _canonical_csc(matrix, n=None):
    m = sparse.csc_matrix(matrix, dtype=np.float64)
    m.sum_duplicates()
    m.sort_indices()
    if n is not None and m.shape != (n, n):
        raise ValueError(f"expected a {n} x {n} matrix, got {m.shape}")
    return m


def _matrix_data(indptr, indices, values, n):
    indptr = np.ascontiguousarray(indptr, np.int64)
    indices = np.ascontiguousarray(indices, np.int64)
    values = np.ascontiguousarray(values, np.float64)
    data = _lib.MatrixData(n, n, int(indices.shape[0]), indptr.ctypes.data_as(_PI64),
                           indices.ctypes.data_as(_PI64), values.ctypes.data_as(_PF64))
    return data, (indptr, indices, values)  # the arrays must outlive the call


def _residual_adjoint_arrays(n, a_indptr, a_indices, a_values, m_indptr, m_indices, m_values, want_grad_m=True,
                             want_grad_a=True, device=-1):
    a_data, keep_a = _matrix_data(a_indptr, a_indices, a_values, n)
    m_data, keep_m = _matrix_data(m_indptr, m_indices, m_values, n)
    loss = ctypes.c_double(0.0)
    grad_m = np.zeros(m_data.nnz, np.float64) if want_grad_m else None
    grad_a = np.zeros(a_data.nnz, np.float64) if want_grad_a else None
    err = _lib.error_buffer()
    rc = _lib.load().spai_residual_adjoint(a_data, m_data, int(device), ctypes.byref(loss),
                                           grad_m.ctypes.data_as(_PF64) if grad_m is not None else None,
                                           grad_a.ctypes.data_as(_PF64) if grad_a is not None else None,
                                           err, len(err))
    del keep_a, keep_m
    if rc != 0:
        raise RuntimeError(err.value.decode("utf-8", "replace"))
    return float(loss.value), grad_m, grad_a


def residual_adjoint(A, M, device=-1):
    """(f, df/dM, df/dA) for f = ||I - A M||_F^2; the gradients are CSC
    matrices with exactly the (canonical) patterns of M and A."""
    A = _canonical_csc(A)
    n = A.shape[0]
    if A.shape[1] != n:
        raise ValueError("A must be square")
    M = _canonical_csc(M, n)
    loss, gm, ga = _residual_adjoint_arrays(n, A.indptr, A.indices, A.data, M.indptr, M.indices, M.data,
                                            device=device)
    grad_m = sparse.csc_matrix((gm, M.indices.copy(), M.indptr.copy()), shape=M.shape)
    grad_a = sparse.csc_matrix((ga, A.indices.copy(), A.indptr.copy()), shape=A.shape)
    return loss, grad_m, grad_a


def pcg_adjoint(a_values, a_indices, a_offsets, m_values, m_indices, m_offsets, x, grad_x, max_iterations,
                tolerance, refresh_period=0, m_precision="fp64", device=-1, symmetric_part=False):
    """Reverse mode of `pcg` on CSR A (symmetric positive definite) and CSR M:
    returns (grad_b, grad_a_values, history, status) where grad_b solves
    A grad_b = grad_x with the forward's settings and
    grad_a_values[q] = -grad_b[i] * x[j] for A's entry q = (i, j)."""
    av = np.ascontiguousarray(a_values, np.float64)
    ai = np.ascontiguousarray(a_indices, np.int64)
    ao = np.ascontiguousarray(a_offsets, np.int64)
    mv = np.ascontiguousarray(m_values, np.float64)
    mi = np.ascontiguousarray(m_indices, np.int64)
    mo = np.ascontiguousarray(m_offsets, np.int64)
    x = np.ascontiguousarray(x, np.float64)
    gx = np.ascontiguousarray(grad_x, np.float64)
    n = gx.shape[0]
    if x.shape[0] != n or ao.shape[0] != n + 1 or mo.shape[0] != n + 1:
        raise ValueError("x, grad_x and the CSR offsets must describe the same n")
    params = _lib.PcgParams(int(max_iterations), float(tolerance), int(refresh_period), M_PRECISIONS[m_precision],
                            int(device), 1 if symmetric_part else 0)
    grad_b = np.zeros(n, np.float64)
    grad_a = np.zeros(ai.shape[0], np.float64)
    history = np.zeros(int(max_iterations), np.float64)
    status = ctypes.c_int64(0)
    err = _lib.error_buffer()
    count = _lib.load().spai_pcg_adjoint(n, av.ctypes.data_as(_PF64), ai.ctypes.data_as(_PI64),
                                         ao.ctypes.data_as(_PI64), mv.ctypes.data_as(_PF64),
                                         mi.ctypes.data_as(_PI64), mo.ctypes.data_as(_PI64),
                                         x.ctypes.data_as(_PF64), gx.ctypes.data_as(_PF64), params,
                                         grad_b.ctypes.data_as(_PF64), grad_a.ctypes.data_as(_PF64),
                                         history.ctypes.data_as(_PF64), ctypes.byref(status), err, len(err))
    if count < 0:
        raise RuntimeError(err.value.decode("utf-8", "replace"))
    return grad_b, grad_a, history[:count].copy(), int(status.value)


def _host(t):
    return t.detach().to("cpu", torch.float64).numpy()


def _on_device(values, device):
    """A contiguous float64 / int64 copy-or-view of `values` on `device`."""
    if isinstance(values, torch.Tensor):
        t = values.detach()
    else:
        t = torch.from_numpy(np.ascontiguousarray(values))
    dtype = torch.float64 if t.is_floating_point() else torch.int64
    return t.to(device=device, dtype=dtype).contiguous()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else None


def _ready(device):
    # the library runs on its own stream: the inputs' producers must be done
    torch.cuda.current_stream(device).synchronize()


def _residual_adjoint_device(n, a_pattern, a_values, m_pattern, m_values, want_m, want_a):
    dev = a_values.device
    if m_values.device != dev:
        raise ValueError("A's and M's values must live on the same device")
    a_ptr, a_idx = _on_device(a_pattern[0], dev), _on_device(a_pattern[1], dev)
    m_ptr, m_idx = _on_device(m_pattern[0], dev), _on_device(m_pattern[1], dev)
    av, mv = _on_device(a_values, dev), _on_device(m_values, dev)
    grad_m = torch.empty(mv.numel(), dtype=torch.float64, device=dev) if want_m else None
    grad_a = torch.empty(av.numel(), dtype=torch.float64, device=dev) if want_a else None
    loss = ctypes.c_double(0.0)
    err = _lib.error_buffer()
    _ready(dev)
    rc = _lib.load().spai_residual_adjoint_device(n, av.numel(), _ptr(a_ptr), _ptr(a_idx), _ptr(av), mv.numel(),
                                                  _ptr(m_ptr), _ptr(m_idx), _ptr(mv), dev.index, ctypes.byref(loss),
                                                  _ptr(grad_m), _ptr(grad_a), err, len(err))
    if rc != 0:
        raise RuntimeError(err.value.decode("utf-8", "replace"))
    return float(loss.value), grad_m, grad_a


class ResidualObjective(torch.autograd.Function):
    """f = ||I - A M||_F^2 over the stored values of A and M (fixed canonical
    CSC patterns, given as (indptr, indices) numpy arrays)."""

    @staticmethod
    def forward(ctx, a_values, m_values, a_pattern, m_pattern, n, device):
        want_m, want_a = ctx.needs_input_grad[1], ctx.needs_input_grad[0]
        if a_values.is_cuda:
            loss, ctx.grad_m, ctx.grad_a = _residual_adjoint_device(n, a_pattern, a_values, m_pattern, m_values,
                                                                    want_m, want_a)
            return torch.tensor(loss, dtype=torch.float64, device=a_values.device)
        loss, gm, ga = _residual_adjoint_arrays(n, a_pattern[0], a_pattern[1], _host(a_values), m_pattern[0],
                                                m_pattern[1], _host(m_values), want_m, want_a, device)
        ctx.grad_m = None if gm is None else torch.from_numpy(gm).to(m_values.device)
        ctx.grad_a = None if ga is None else torch.from_numpy(ga).to(a_values.device)
        return torch.tensor(loss, dtype=torch.float64, device=a_values.device)

    @staticmethod
    def backward(ctx, grad_loss):
        grad_a = None if ctx.grad_a is None else grad_loss * ctx.grad_a
        grad_m = None if ctx.grad_m is None else grad_loss * ctx.grad_m
        return grad_a, grad_m, None, None, None, None


def residual_objective(a_values, m_values, a_pattern, m_pattern, device=-1):
    """Differentiable ||I - A M||_F^2.  a_pattern / m_pattern: (indptr, indices)
    of canonical n x n CSC patterns; a_values / m_values: float64 tensors of
    their stored values."""
    n = len(a_pattern[0]) - 1
    if len(m_pattern[0]) - 1 != n:
        raise ValueError("A and M must have the same size")
    return ResidualObjective.apply(a_values, m_values, a_pattern, m_pattern, n, device)


class PcgSolve(torch.autograd.Function):
    """x = A^-1 b by the device PCG; gradients for A's stored values (CSR,
    fixed pattern) and b through `pcg_adjoint`."""

    @staticmethod
    def forward(ctx, a_values, b, a_pattern, m_csr, options):
        a_indices, a_offsets = a_pattern
        m_values, m_indices, m_offsets = m_csr
        if a_values.is_cuda:
            return PcgSolve._forward_device(ctx, a_values, b, a_pattern, m_csr, options)
        av = _host(a_values)
        history, status, x = pcg(av, a_indices, a_offsets, m_values, m_indices, m_offsets, _host(b),
                                 options["max_iterations"], 1, options["tolerance"],
                                 refresh_period=options.get("refresh_period", 0),
                                 m_precision=options.get("m_precision", "fp64"), device=options.get("device", -1),
                                 return_x=True, symmetric_part=options.get("symmetric_part", False))
        ctx.state = (av, a_pattern, m_csr, options, x)
        ctx.history, ctx.status = history, status
        return torch.from_numpy(x).to(b.device)

    @staticmethod
    def _params(options, device):
        return _lib.PcgParams(int(options["max_iterations"]), float(options["tolerance"]),
                              int(options.get("refresh_period", 0)), M_PRECISIONS[options.get("m_precision", "fp64")],
                              int(device), 1 if options.get("symmetric_part", False) else 0)

    @staticmethod
    def _forward_device(ctx, a_values, b, a_pattern, m_csr, options):
        dev = a_values.device
        if b.device != dev:
            raise ValueError("A's values and b must live on the same device")
        av, bv = _on_device(a_values, dev), _on_device(b, dev)
        ai, ao = _on_device(a_pattern[0], dev), _on_device(a_pattern[1], dev)
        mv, mi, mo = (_on_device(v, dev) for v in m_csr)
        n = bv.numel()
        if ao.numel() != n + 1 or mo.numel() != n + 1:
            raise ValueError("b and the CSR offsets must describe the same n")
        x = torch.empty(n, dtype=torch.float64, device=dev)
        history = np.zeros(int(options["max_iterations"]), np.float64)
        status = ctypes.c_int64(0)
        err = _lib.error_buffer()
        _ready(dev)
        count = _lib.load().spai_pcg_device(n, av.numel(), _ptr(av), _ptr(ai), _ptr(ao), mv.numel(), _ptr(mv),
                                            _ptr(mi), _ptr(mo), _ptr(bv), PcgSolve._params(options, dev.index),
                                            history.ctypes.data_as(_PF64), ctypes.byref(status), _ptr(x), err,
                                            len(err))
        if count < 0:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        ctx.device_state = (av, ai, ao, mv, mi, mo, x, options)
        ctx.history, ctx.status = history[:count].copy(), int(status.value)
        return x

    @staticmethod
    def _backward_device(ctx, grad_x):
        av, ai, ao, mv, mi, mo, x, options = ctx.device_state
        dev = x.device
        gx = _on_device(grad_x, dev)
        n = x.numel()
        grad_b = torch.empty(n, dtype=torch.float64, device=dev)
        grad_a = torch.empty(av.numel(), dtype=torch.float64, device=dev)
        history = np.zeros(int(options["max_iterations"]), np.float64)
        status = ctypes.c_int64(0)
        err = _lib.error_buffer()
        _ready(dev)
        count = _lib.load().spai_pcg_adjoint_device(n, av.numel(), _ptr(av), _ptr(ai), _ptr(ao), mv.numel(),
                                                    _ptr(mv), _ptr(mi), _ptr(mo), _ptr(x), _ptr(gx),
                                                    PcgSolve._params(options, dev.index), _ptr(grad_b), _ptr(grad_a),
                                                    history.ctypes.data_as(_PF64), ctypes.byref(status), err, len(err))
        if count < 0:
            raise RuntimeError(err.value.decode("utf-8", "replace"))
        return grad_a, grad_b, None, None, None

    @staticmethod
    def backward(ctx, grad_x):
        if getattr(ctx, "device_state", None) is not None:
            return PcgSolve._backward_device(ctx, grad_x)
        av, (a_indices, a_offsets), (m_values, m_indices, m_offsets), options, x = ctx.state
        grad_b, grad_a, _, _ = pcg_adjoint(av, a_indices, a_offsets, m_values, m_indices, m_offsets, x,
                                           _host(grad_x), options["max_iterations"], options["tolerance"],
                                           refresh_period=options.get("refresh_period", 0),
                                           m_precision=options.get("m_precision", "fp64"),
                                           device=options.get("device", -1),
                                           symmetric_part=options.get("symmetric_part", False))
        device = grad_x.device
        return torch.from_numpy(grad_a).to(device), torch.from_numpy(grad_b).to(device), None, None, None


def pcg_solve(a_values, b, a_indices, a_offsets, m_values, m_indices, m_offsets, max_iterations=1000,
              tolerance=1e-10, **options):
    """Differentiable PCG solve: x = A^-1 b for CSR A (pattern fixed, values
    a float64 tensor) preconditioned by CSR M (numpy arrays, constant)."""
    opts = dict(options, max_iterations=int(max_iterations), tolerance=float(tolerance))
    a_pattern = (np.ascontiguousarray(a_indices, np.int64), np.ascontiguousarray(a_offsets, np.int64))
    m_csr = (np.ascontiguousarray(m_values, np.float64), np.ascontiguousarray(m_indices, np.int64),
             np.ascontiguousarray(m_offsets, np.int64))
    return PcgSolve.apply(a_values, b, a_pattern, m_csr, opts)
