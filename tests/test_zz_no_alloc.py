"""spai_pcg_device_noalloc, the allocation-free PCG on device buffers, against
spai_pcg (the host-buffer entry point with the same arithmetic).

The file name sorts last so that, in a full run, the entry point is exercised
after every other test has used the library in the same process; it must also
pass alone in a fresh process.  Both entry points compute the same bits, so
the tolerance is zero.
"""
import ctypes
import json
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest
from scipy import sparse

from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib, backward_error, problems

MAX_ROWS = 524_288


def _polynomial_preconditioner(a):
    """D^-1/2 (2I - D^-1/2 A D^-1/2) D^-1/2 as CSR: symmetric, sparse, cheap."""
    d = sparse.diags(1.0 / np.sqrt(a.diagonal()))
    s = d @ a @ d
    m = sparse.csr_matrix(d @ (2.0 * sparse.identity(a.shape[0]) - s) @ d)
    m.sum_duplicates()
    m.sort_indices()
    return m


def _on_device(torch, m):
    m = sparse.csr_matrix(m)
    return (m.nnz, torch.tensor(m.data, dtype=torch.float64, device="cuda"),
            torch.tensor(m.indices.astype(np.int32), device="cuda"),
            torch.tensor(m.indptr.astype(np.int64), device="cuda"))


def _noalloc(torch, a_dev, m_dev, b_dev, x_dev, max_iterations, tolerance, refresh_period, stream=None):
    lib = _lib.load()
    history = np.full(max_iterations, np.nan)
    status = ctypes.c_int64(-7)
    err = ctypes.create_string_buffer(512)
    a_nnz, av, ai, ao = a_dev
    m_nnz, mv, mi, mo = m_dev
    count = lib.spai_pcg_device_noalloc(
        b_dev.numel(), a_nnz, av.data_ptr(), ai.data_ptr(), ao.data_ptr(), m_nnz, mv.data_ptr(), mi.data_ptr(),
        mo.data_ptr(), b_dev.data_ptr(), x_dev.data_ptr(), max_iterations, tolerance, refresh_period, stream,
        history.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(status), err, len(err))
    assert count > 0, err.value.decode()
    return history[:count], int(status.value), x_dev.cpu().numpy()


def _spai_pcg(a, m, b, max_iterations, tolerance, refresh_period):
    a = sparse.csr_matrix(a)
    a.sort_indices()
    return backward_error.pcg(a.data, a.indices, a.indptr, m.data, m.indices, m.indptr, b, max_iterations, 1,
                              tolerance, refresh_period=refresh_period, m_precision="fp64", return_x=True)


CASES = {
    # one tree chunk (n <= 4096)
    "laplacian_2d_64": (lambda: problems.laplacian_2d(64), 400, 1e-8, 0),
    # many tree chunks, periodic true-residual refresh
    "diffusion_3d_40": (lambda: problems.diffusion_3d(40, 1.0, 3), 400, 1e-8, 7),
    # exactly the largest accepted size
    "tridiagonal_max": (lambda: problems.tridiagonal(MAX_ROWS), 40, 1e-10, 0),
}


@pytest.mark.gpu
def test_noalloc_matches_spai_pcg_on_consecutive_calls(require_gpu):
    import torch
    for label, (maker, iters, tol, refresh) in CASES.items():
        a = sparse.csr_matrix(maker())
        a.sort_indices()
        m = _polynomial_preconditioner(a)
        b, _ = problems.solution_rhs(a, seed=5)
        want_h, want_s, want_x = _spai_pcg(a, m, b, iters, tol, refresh)
        a_dev, m_dev = _on_device(torch, a), _on_device(torch, m)
        b_dev = torch.tensor(b, dtype=torch.float64, device="cuda")
        # two calls in a row: the default stream, then a side stream
        x1 = torch.full_like(b_dev, 3.0)
        got1 = _noalloc(torch, a_dev, m_dev, b_dev, x1, iters, tol, refresh)
        side = torch.cuda.Stream()
        torch.cuda.synchronize()
        x2 = torch.full_like(b_dev, -1.0)
        got2 = _noalloc(torch, a_dev, m_dev, b_dev, x2, iters, tol, refresh, stream=side.cuda_stream)
        for got in (got1, got2):
            h, s, x = got
            np.testing.assert_array_equal(h, want_h, err_msg=f"{label} history")
            assert s == want_s, label
            np.testing.assert_array_equal(x, want_x, err_msg=f"{label} x")
        assert len(want_h) > 2, label


@pytest.mark.gpu
def test_noalloc_rejects_host_pointers_and_bad_csr(require_gpu):
    import torch
    a = sparse.csr_matrix(problems.laplacian_2d(8))
    a.sort_indices()
    m = _polynomial_preconditioner(a)
    a_dev, m_dev = _on_device(torch, a), _on_device(torch, m)
    b = np.ones(a.shape[0])
    x_dev = torch.zeros(a.shape[0], dtype=torch.float64, device="cuda")
    lib = _lib.load()
    err = ctypes.create_string_buffer(512)
    history = np.zeros(10)
    status = ctypes.c_int64(0)

    def call(a_arrays, b_ptr, n=a.shape[0]):
        a_nnz, av, ai, ao = a_arrays
        m_nnz, mv, mi, mo = m_dev
        return lib.spai_pcg_device_noalloc(n, a_nnz, av.data_ptr(), ai.data_ptr(), ao.data_ptr(), m_nnz,
                                           mv.data_ptr(), mi.data_ptr(), mo.data_ptr(), b_ptr, x_dev.data_ptr(),
                                           10, 1e-8, 0, None, history.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                           ctypes.byref(status), err, len(err))

    # b in host memory: refused before any kernel runs
    assert call(a_dev, b.ctypes.data) == -1
    assert b"device memory" in err.value
    b_dev = torch.tensor(b, device="cuda")
    # a column index outside [0, n): found by the device-side check, no SpMV runs
    bad_idx = a_dev[2].clone()
    bad_idx[5] = a.shape[0] + 3
    assert call((a_dev[0], a_dev[1], bad_idx, a_dev[3]), b_dev.data_ptr()) == -1
    assert b"malformed CSR input (A)" in err.value
    # x may not alias an input: x is cleared before r = b is formed
    alias = lib.spai_pcg_device_noalloc(a.shape[0], a_dev[0], a_dev[1].data_ptr(), a_dev[2].data_ptr(),
                                        a_dev[3].data_ptr(), m_dev[0], m_dev[1].data_ptr(), m_dev[2].data_ptr(),
                                        m_dev[3].data_ptr(), b_dev.data_ptr(), b_dev.data_ptr(), 10, 1e-8, 0, None,
                                        history.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(status),
                                        err, len(err))
    assert alias == -1
    assert b"x overlaps b" in err.value
    # the valid call still works afterwards
    assert call(a_dev, b_dev.data_ptr()) > 1, err.value.decode()


# A child process without torch: the runtime's own allocator holds the
# buffers, so that cudaDeviceReset (which ends this process's context on the
# device) leaves no other library state behind.  Only the no-alloc entry
# point runs, before and after the reset.
_RESET_CHILD = textwrap.dedent("""
    import ctypes, json, sys
    import numpy as np
    from scipy import sparse
    sys.path.insert(0, sys.argv[1])
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib, problems
    lib = _lib.load()
    rt = ctypes.CDLL("libcudart.so.12")
    def ok(rc, what):
        if rc != 0:
            raise SystemExit(f"{what}: cuda error {rc}")
    ok(rt.cudaSetDevice(0), "cudaSetDevice")
    a = sparse.csr_matrix(problems.diffusion_3d(24, 1.0, 2))
    a.sort_indices()
    d = sparse.diags(1.0 / np.sqrt(a.diagonal()))
    m = sparse.csr_matrix(d @ (2.0 * sparse.identity(a.shape[0]) - d @ a @ d) @ d)
    m.sum_duplicates()
    m.sort_indices()
    b, _ = problems.solution_rhs(a, seed=5)
    n = a.shape[0]
    def upload(arr):
        arr = np.ascontiguousarray(arr)
        ptr = ctypes.c_void_p()
        ok(rt.cudaMalloc(ctypes.byref(ptr), ctypes.c_size_t(max(arr.nbytes, 8))), "cudaMalloc")
        ok(rt.cudaMemcpy(ptr, arr.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(arr.nbytes), 1), "H2D")
        return ptr
    def solve():
        bufs = [upload(x) for x in (a.data, a.indices.astype(np.int32), a.indptr.astype(np.int64), m.data,
                                    m.indices.astype(np.int32), m.indptr.astype(np.int64), b, np.zeros(n))]
        history = np.full(300, np.nan)
        status = ctypes.c_int64(-7)
        err = ctypes.create_string_buffer(512)
        count = lib.spai_pcg_device_noalloc(n, a.nnz, bufs[0], bufs[1], bufs[2], m.nnz, bufs[3], bufs[4], bufs[5],
                                            bufs[6], bufs[7], 300, 1e-9, 11, None,
                                            history.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            ctypes.byref(status), err, len(err))
        if count < 0:
            raise SystemExit("noalloc: " + err.value.decode())
        x = np.empty(n)
        ok(rt.cudaMemcpy(x.ctypes.data_as(ctypes.c_void_p), bufs[7], ctypes.c_size_t(x.nbytes), 2), "D2H")
        for ptr in bufs:
            ok(rt.cudaFree(ptr), "cudaFree")
        return history[:count], int(status.value), x
    h1, s1, x1 = solve()
    ok(rt.cudaDeviceReset(), "cudaDeviceReset")
    ok(rt.cudaSetDevice(0), "cudaSetDevice")
    h2, s2, x2 = solve()
    print(json.dumps({"len": len(h1), "status": [s1, s2],
                      "same_history": bool(np.array_equal(h1.view(np.int64), h2.view(np.int64))),
                      "same_x": bool(np.array_equal(x1.view(np.int64), x2.view(np.int64)))}))
""")


@pytest.mark.gpu
def test_noalloc_after_device_reset_gives_the_same_bits(require_gpu):
    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0])
    proc = subprocess.run([sys.executable, "-c", _RESET_CHILD, str(root)], capture_output=True, text=True,
                          timeout=300, env=env)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    out = json.loads(proc.stdout.strip().splitlines()[-1])
    assert out["len"] > 2 and out["status"][0] == out["status"][1] == 1, out
    assert out["same_history"] and out["same_x"], out


def test_noalloc_rejects_oversize_before_touching_the_device():
    lib = _lib.load()
    err = ctypes.create_string_buffer(256)
    history = np.zeros(4)
    status = ctypes.c_int64(0)
    count = lib.spai_pcg_device_noalloc(MAX_ROWS + 1, 0, None, None, None, 0, None, None, None, None, None, 4,
                                        1e-8, 0, None, history.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        ctypes.byref(status), err, len(err))
    assert count == -1
    assert b"524288" in err.value
