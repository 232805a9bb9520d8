"""GPU PCG against the oracle PCG in the device order (bit-identical history
and status) and against the reference's own PCG (iteration counts within 1)."""
import numpy as np
import pytest
from scipy import sparse

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import backward_error, problems

pytestmark = pytest.mark.gpu


def _csr(m):
    m = sparse.csr_matrix(m)
    m.sort_indices()
    return m


@pytest.mark.parametrize("tolerance", [1e-6, 1e-8])
@pytest.mark.parametrize("refresh", [0, 7])
def test_pcg_matches_oracle(require_gpu, tolerance, refresh):
    A = _csr(problems.diffusion_2d(24, 1.0, 5))
    M = _csr(problems.diagonal_inverse(A))
    b, _ = problems.solution_rhs(A, seed=0)
    hist, status = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, b, 2000, 1,
                                      tolerance, refresh_period=refresh)
    want, want_status = pyoracle.pcg(A, M, b, 2000, tolerance, order=pyoracle.ORDER_DEVICE, refresh_period=refresh)
    assert status == want_status == 1
    assert np.array_equal(hist.view(np.int64), want.view(np.int64))


def test_pcg_mixed_m_close_to_fp64(require_gpu):
    A = _csr(problems.diffusion_2d(24, 1.0, 5))
    M = _csr(problems.diagonal_inverse(A))
    b, _ = problems.solution_rhs(A, seed=0)
    h64, s64 = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, b, 2000, 1, 1e-8)
    h32, s32 = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, b, 2000, 1, 1e-8,
                                  m_precision="mixed")
    assert s64 == s32 == 1
    assert abs(len(h64) - len(h32)) <= 2
    assert h32[-1] <= 1e-8


def test_matvec_matches_scipy(require_gpu):
    A = _csr(problems.diffusion_2d(20, 1.0, 1))
    x = np.random.default_rng(3).standard_normal(A.shape[0])
    y = backward_error.matvec(A.data, A.indices, A.indptr, x, 1)
    assert np.allclose(y, A @ x, rtol=1e-14, atol=1e-14)
