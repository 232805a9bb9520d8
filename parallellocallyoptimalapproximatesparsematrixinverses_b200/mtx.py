"""Matrix Market files through libspai_b200.so's native reader and writer
(`spai_mtx_read` / `spai_mtx_write`), mirroring how the reference's drivers
use scipy.io:

* `load_matrix(path)`: the canonical CSC of scripts/common.py:397-402
  (mmread, tocsc, float64, sum_duplicates, eliminate_zeros, sort_indices);
* `save_preconditioner(dataset_dir, method_name, M)`:
  <dataset_dir>/<method_name>/preconditioner.mtx (scripts/common.py:494-500);
* `load_preconditioner(path)`: CSR float64 (scripts/utils/backward_error.py:111-113).

The reader parses on all host threads and needs no scipy round trip; values
are written with 17 significant digits, so a saved M reads back bit for bit.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np
from scipy import sparse

from . import _lib
from .methods import adopt_matrix, as_csc, matrix_data


def load_matrix(path, threads: int = 0) -> sparse.csc_matrix:
    """Canonical float64 CSC of a Matrix Market file (int64 indices)."""
    lib = _lib.load()
    result = lib.spai_mtx_read(os.fsencode(Path(path)), int(threads))
    try:
        if result.error_message:
            raise RuntimeError(result.error_message.decode("utf-8", "replace"))
        m = adopt_matrix(result)
        m.has_sorted_indices = True
        return m
    finally:
        lib.free_mem(ctypes.byref(result))


def write_matrix(path, M, symmetric: bool = False) -> Path:
    """Writes M as a coordinate real Matrix Market file (lower triangle only
    when `symmetric`)."""
    path = Path(path)
    csc = as_csc(M)
    err = _lib.error_buffer()
    rc = _lib.load().spai_mtx_write(os.fsencode(path), matrix_data(csc), 1 if symmetric else 0, err, len(err))
    if rc != 0:
        raise RuntimeError(err.value.decode("utf-8", "replace"))
    return path


def save_preconditioner(dataset_dir, method_name: str, M) -> Path:
    """<dataset_dir>/<method_name>/preconditioner.mtx, as the reference's
    _save_preconditioner_matrix lays it out."""
    method_dir = Path(dataset_dir) / method_name
    method_dir.mkdir(parents=True, exist_ok=True)
    return write_matrix(method_dir / "preconditioner.mtx", M)


def load_preconditioner(path) -> sparse.csr_matrix:
    """A saved preconditioner as CSR float64 (the form PCG takes)."""
    return sparse.csr_matrix(load_matrix(path), dtype=np.float64)
