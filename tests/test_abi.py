"""The C ABI without a GPU: the library loads, exports every function that
include/*.h declares, keeps the reference's struct layout, and reports the
reference's validation errors before touching the device."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest
from scipy import sparse

from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib, global_spai, inner_outer, problems
from tests.conftest import cuda_available

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_functions():
    names = set()
    for header in INCLUDE.glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            prefix = text[:m.start()].rstrip()
            if name in {"if", "for", "while", "sizeof", "return"} or prefix.endswith("#define"):
                continue
            if re.search(r"(Result|void|int64_t|SpaiSession\s*\*|void\s*\*)\s*$", prefix):
                names.add(name)
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    declared = declared_functions()
    assert "spai_global_mr" in declared and "free_mem" in declared
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/*.h but not exported"
    assert set(declared) <= set(_lib.EXPORTED_SYMBOLS)


def test_struct_layout_matches_reference():
    # reference include/methods_c_api.h:7-46: every field is 8 bytes
    assert ctypes.sizeof(_lib.MatrixData) == 48
    assert ctypes.sizeof(_lib.MethodParams) == 64
    assert ctypes.sizeof(_lib.SingleIterationData) == 32
    assert ctypes.sizeof(_lib.Result) == 88


def test_free_mem_nulls_pointers():
    lib = _lib.load()
    r = _lib.Result()
    lib.free_mem(ctypes.byref(r))
    lib.free_mem(None)
    assert not r.col_offsets and not r.error_message


def _raw_call(A, **overrides):
    lib = _lib.load()
    csc = sparse.csc_matrix(A)
    indptr = np.ascontiguousarray(csc.indptr, np.int64)
    indices = np.ascontiguousarray(csc.indices, np.int64)
    data = np.ascontiguousarray(csc.data, np.float64)
    md = _lib.MatrixData(csc.shape[0], csc.shape[1], csc.nnz, indptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    for k, v in overrides.items():
        setattr(md, k, v)
    params = _lib.MethodParams(10, 1e-9, 1.0, 1, 1, 0, 0, 2)
    empty = _lib.MatrixData()
    res = lib.spai_global_mr(md, empty, empty, params)
    msg = res.error_message.decode() if res.error_message else None
    lib.free_mem(ctypes.byref(res))
    return msg, (indptr, indices, data)


def test_validation_messages_match_reference():
    A = problems.tridiagonal(12)
    msg, _ = _raw_call(A, nnz=0)
    assert msg == "Sparse matrix dimensions and nnz must be positive"
    csc = sparse.csc_matrix(A)
    bad = np.ascontiguousarray(csc.indices, np.int64).copy()
    bad[3] = 99
    lib = _lib.load()
    indptr = np.ascontiguousarray(csc.indptr, np.int64)
    data = np.ascontiguousarray(csc.data)
    md = _lib.MatrixData(12, 12, csc.nnz, indptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         bad.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    res = lib.spai_global_mr(md, _lib.MatrixData(), _lib.MatrixData(), _lib.MethodParams(10, 1e-9, 1.0, 1, 1, 0, 0, 2))
    assert res.error_message.decode() == "Sparse matrix row idx is out of range"
    lib.free_mem(ctypes.byref(res))
    with pytest.raises(RuntimeError, match="max_iterations must be positive"):
        global_spai.mr(A, max_iterations=0, max_density=1.0)
    with pytest.raises(RuntimeError, match="tolerance must be finite and non-negative"):
        global_spai.cg(A, tolerance=-1.0, max_density=1.0)
    with pytest.raises(RuntimeError, match=r"max_density must be finite and in the interval \(0, 1\]"):
        global_spai.lomr(A, max_density=1.5)
    with pytest.raises(RuntimeError, match="max_density is too small to preserve the diagonal of M"):
        global_spai.mr(A)
    with pytest.raises(RuntimeError, match="Invalid threads count value"):
        global_spai.mr(A, max_density=1.0, num_threads=0)
    with pytest.raises(RuntimeError, match="inner_iterations must be positive"):
        inner_outer.mr(A, max_density=1.0, inner_iterations=0)
    with pytest.raises(RuntimeError, match="Initial preconditioner M0 must have the same shape as A"):
        _raw_shape_mismatch(A)


def _raw_shape_mismatch(A):
    lib = _lib.load()
    csc = sparse.csc_matrix(A)
    indptr = np.ascontiguousarray(csc.indptr, np.int64)
    indices = np.ascontiguousarray(csc.indices, np.int64)
    data = np.ascontiguousarray(csc.data)
    md = _lib.MatrixData(12, 12, csc.nnz, indptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         data.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    m0 = sparse.identity(5, format="csc")
    p0 = np.ascontiguousarray(m0.indptr, np.int64)
    i0 = np.ascontiguousarray(m0.indices, np.int64)
    d0 = np.ascontiguousarray(m0.data)
    m0d = _lib.MatrixData(5, 5, 5, p0.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                          i0.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                          d0.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    res = lib.spai_global_mr(md, m0d, _lib.MatrixData(), _lib.MethodParams(10, 1e-9, 1.0, 1, 1, 1, 0, 2))
    msg = res.error_message.decode() if res.error_message else ""
    lib.free_mem(ctypes.byref(res))
    raise RuntimeError(msg)


@pytest.mark.skipif(cuda_available(), reason="checks the behaviour on a host without a GPU")
def test_no_silent_cpu_fallback():
    with pytest.raises(RuntimeError, match="no CUDA device"):
        global_spai.mr(problems.tridiagonal(12), max_density=1.0)
