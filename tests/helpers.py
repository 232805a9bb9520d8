"""Helpers shared by the tests: method tables and result comparison."""
from __future__ import annotations

import numpy as np
from scipy import sparse

METHODS = [
    ("global_spai", "cg"),
    ("global_spai", "mr"),
    ("global_spai", "lomr"),
    ("inner_outer", "mr"),
    ("inner_outer", "lomr"),
]


def bit_equal(a, b) -> bool:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def assert_same_result(got, want, context=""):
    """Bit-exact equality of two OutputResult objects (M pattern, M values, history)."""
    assert got.iterations == want.iterations, f"{context}: iterations {got.iterations} != {want.iterations}"
    assert got.converged == want.converged, f"{context}: converged differs"
    gh, wh = got.history, want.history
    assert gh.shape == wh.shape, f"{context}: history length {gh.shape} != {wh.shape}"
    assert np.array_equal(gh["iteration"], wh["iteration"]), context
    for field in ("residual_norm", "density_m", "density_direction"):
        if not bit_equal(gh[field], wh[field]):
            bad = np.nonzero(gh[field] != wh[field])[0]
            raise AssertionError(f"{context}: history {field} differs first at row {bad[:3]}: "
                                 f"{gh[field][bad[:3]]} vs {wh[field][bad[:3]]}")
    gm = sparse.csc_matrix(got.M)
    wm = sparse.csc_matrix(want.M)
    assert gm.shape == wm.shape, context
    assert np.array_equal(gm.indptr, wm.indptr), f"{context}: column pointers differ"
    assert np.array_equal(gm.indices, wm.indices), f"{context}: row indices differ"
    if not bit_equal(gm.data, wm.data):
        diff = np.abs(gm.data - wm.data) / np.maximum(np.abs(wm.data), 1e-300)
        raise AssertionError(f"{context}: M values differ, max rel {diff.max():.3e}")


def relative_difference(got, want) -> float:
    d = sparse.csc_matrix(got) - sparse.csc_matrix(want)
    denom = sparse.linalg.norm(want)
    return float(sparse.linalg.norm(d) / denom) if denom > 0 else float(sparse.linalg.norm(d))
