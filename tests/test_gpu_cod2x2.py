"""The device's 2x2 minimum-norm least-squares solve (cod2x2.cuh, the
per-column Inner-Outer LOMR step; reference src/common/sparse_operations.cpp:58-73)
against the oracle's independent restatement, bit for bit, on the branches a
LOMR run rarely reaches: full rank, rank one, near-singular, zero, and
non-finite inputs or outputs."""
import ctypes

import numpy as np
import pytest

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib

pytestmark = pytest.mark.gpu

_PF64 = ctypes.POINTER(ctypes.c_double)


def _cases():
    rng = np.random.default_rng(21)
    cases = [
        ([[4.0, 1.0], [1.0, 3.0]], [1.0, 2.0]),              # full rank
        ([[1.0, 2.0], [2.0, 4.0]], [1.0, 2.0]),              # rank one, consistent
        ([[1.0, 2.0], [2.0, 4.0]], [1.0, -3.0]),             # rank one, inconsistent
        ([[1.0, 1.0], [1.0, 1.0 + 1e-15]], [2.0, 2.0]),      # near-singular below the rank threshold
        ([[1.0, 1.0], [1.0, 1.0 + 1e-9]], [2.0, 1.0]),       # near-singular above it
        ([[2.0, 0.0], [0.0, 0.0]], [1.0, 1.0]),              # a zero diagonal entry
        ([[0.0, 0.0], [0.0, 0.0]], [1.0, 1.0]),              # all zero
        ([[-3.0, 1.0], [1.0, -2.0]], [0.5, 0.25]),           # negative diagonal (scaled by 1/sqrt|m_ii|)
        ([[1e-300, 0.0], [0.0, 1e300]], [1.0, 1.0]),         # extreme scales
        ([[np.nan, 0.0], [0.0, 1.0]], [1.0, 1.0]),           # NaN input
        ([[1.0, 0.0], [0.0, 1.0]], [np.inf, 1.0]),           # Inf input
        ([[np.inf, 1.0], [1.0, 1.0]], [1.0, 1.0]),           # Inf in the matrix
        ([[1e-308, 1e-308], [1e-308, 1e-308]], [1e308, 1e308]),  # overflowing solution
    ]
    for _ in range(40):
        a = rng.standard_normal((2, 2)) * 10.0 ** rng.integers(-6, 6)
        m = a @ a.T
        if rng.random() < 0.5:
            m[1] = m[0] * rng.uniform(-3, 3)  # singular
            m[:, 1] = m[1]
        cases.append((m.tolist(), (rng.standard_normal(2) * 10.0 ** rng.integers(-3, 3)).tolist()))
    return cases


def test_device_2x2_solve_matches_the_oracle(require_gpu):
    cases = _cases()
    gram = np.ascontiguousarray([np.array(m, dtype=np.float64).reshape(4) for m, _ in cases])
    rhs = np.ascontiguousarray([np.array(r, dtype=np.float64) for _, r in cases])
    out = np.full((len(cases), 2), np.nan)
    err = ctypes.create_string_buffer(256)
    lib = _lib.load()
    rc = lib.spai_solve_2x2_device(len(cases), gram.ctypes.data_as(_PF64), rhs.ctypes.data_as(_PF64),
                                   out.ctypes.data_as(_PF64), err, len(err))
    assert rc == 0, err.value.decode()
    for i, (m, r) in enumerate(cases):
        want = pyoracle.solve_2x2(m, r)
        assert np.array_equal(out[i].view(np.int64), np.asarray(want).view(np.int64)), (i, m, r, out[i], want)
    # the degenerate branches return zeros, as the reference's guard does
    assert np.array_equal(out[6], [0.0, 0.0]) and np.array_equal(out[9], [0.0, 0.0])
    assert np.array_equal(out[10], [0.0, 0.0])
