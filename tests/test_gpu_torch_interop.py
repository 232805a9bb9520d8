"""Sessions on torch sparse CSC tensors in GPU memory (spai_session_create_device
/ spai_session_result_device): the same M and history as the host entry
points, bit for bit, with no host copy of A, M0 or M; bad device input is
refused from the device-side checks."""
import ctypes

import numpy as np
import pytest
from scipy import sparse

from parallellocallyoptimalapproximatesparsematrixinverses_b200 import Session, _lib, global_spai, inner_outer, problems
from tests.helpers import bit_equal

pytestmark = pytest.mark.gpu
FAMILIES = {"global_spai": global_spai, "inner_outer": inner_outer}


def _torch_csc(torch, m):
    m = sparse.csc_matrix(m)
    m.sort_indices()
    return torch.sparse_csc_tensor(torch.tensor(m.indptr, dtype=torch.int64), torch.tensor(m.indices, dtype=torch.int64),
                                   torch.tensor(m.data, dtype=torch.float64), size=m.shape, device="cuda")


@pytest.mark.parametrize("family,name,precision,topk", [("global_spai", "mr", "fp64", 5),
                                                         ("global_spai", "lomr", "mixed", 6),
                                                         ("inner_outer", "mr", "fp64", 4),
                                                         ("global_spai", "cg", "fp64", 0)])
def test_device_session_matches_host_entry_points(require_gpu, family, name, precision, topk):
    import torch
    A = problems.diffusion_2d(18, 1.0, 3)
    M0 = problems.diagonal_inverse(A)
    kw = dict(max_iterations=6, tolerance=1e-12, max_density=0.05, precision=precision, topk_per_column=topk,
              summation="device")
    want = getattr(FAMILIES[family], name)(A, M0=M0, **kw)
    s = Session.from_torch(family, name, _torch_csc(torch, A), M0=_torch_csc(torch, M0), **kw)
    iterations, nnz = s.run()
    M = s.result_torch()
    assert M.is_cuda and M.layout == torch.sparse_csc
    assert iterations == want.iterations and nnz == want.M.nnz and s.converged == want.converged
    assert np.array_equal(M.ccol_indices().cpu().numpy(), want.M.indptr)
    assert np.array_equal(M.row_indices().cpu().numpy(), want.M.indices)
    assert bit_equal(M.values().cpu().numpy(), want.M.data)
    h = s.history()
    assert bit_equal(h["residual_norm"], want.history["residual_norm"])
    s.close()


def test_device_session_identity_m0_and_pcg(require_gpu):
    import torch
    A = problems.laplacian_2d(16)
    want = global_spai.mr(A, max_iterations=4, tolerance=1e-12, max_density=1.0, topk_per_column=5)
    s = Session.from_torch("global_spai", "mr", _torch_csc(torch, A), max_iterations=4, tolerance=1e-12,
                           max_density=1.0, topk_per_column=5)
    s.run()
    assert bit_equal(s.result_torch().values().cpu().numpy(), want.M.data)
    b, _ = problems.solution_rhs(A, seed=1)
    s.set_rhs(b)
    hist, status = s.pcg(500, 1e-8, symmetric_part=True)
    assert status == 1


def test_device_session_refuses_bad_input(require_gpu):
    import torch
    A = sparse.csc_matrix(problems.laplacian_2d(6))
    A.sort_indices()
    ptr = torch.tensor(A.indptr, dtype=torch.int64, device="cuda")
    rows = torch.tensor(A.indices, dtype=torch.int64, device="cuda")
    vals = torch.tensor(A.data, dtype=torch.float64, device="cuda")
    lib = _lib.load()
    params = _lib.MethodParams(4, 1e-8, 1.0, 0, 1, 0, 0, 2)
    err = ctypes.create_string_buffer(256)

    def create(p, r, v):
        return lib.spai_session_create_device(1, A.shape[0], A.nnz, p, r, v, 0, None, None, None, params, None, err,
                                              len(err))

    unsorted = rows.clone()
    unsorted[[0, 1]] = unsorted[[1, 0]]
    torch.cuda.synchronize()
    assert not create(ptr.data_ptr(), unsorted.data_ptr(), vals.data_ptr())
    assert b"increase strictly" in err.value
    bad_ptr = ptr.clone()
    bad_ptr[-1] = A.nnz - 1
    torch.cuda.synchronize()
    assert not create(bad_ptr.data_ptr(), rows.data_ptr(), vals.data_ptr())
    assert b"from 0 to nnz" in err.value
    host = np.ascontiguousarray(A.indptr, dtype=np.int64)
    assert not create(host.ctypes.data, rows.data_ptr(), vals.data_ptr())
    assert b"device memory" in err.value
    handle = create(ptr.data_ptr(), rows.data_ptr(), vals.data_ptr())
    assert handle, err.value
    lib.spai_session_destroy(handle)
