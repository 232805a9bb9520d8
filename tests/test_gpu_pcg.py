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


def test_pcg_symmetric_part_of_the_transpose_is_the_same(require_gpu):
    # CSC arrays of M read as CSR are M^T; with symmetric_part the preconditioner
    # (M + M^T)/2 is the same either way, bit for bit
    A = _csr(problems.diffusion_2d(20, 1.0, 8))
    rng = np.random.default_rng(4)
    M = sparse.csr_matrix(problems.diagonal_inverse(A) + 0.01 * sparse.random(A.shape[0], A.shape[0], 0.01,
                                                                               random_state=rng))
    M.sort_indices()
    Mc = sparse.csc_matrix(M)
    Mc.sort_indices()
    b, _ = problems.solution_rhs(A, seed=2)
    h1, s1 = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, b, 500, 1, 1e-8,
                                symmetric_part=True)
    h2, s2 = backward_error.pcg(A.data, A.indices, A.indptr, Mc.data, Mc.indices, Mc.indptr, b, 500, 1, 1e-8,
                                symmetric_part=True)
    assert s1 == s2 and np.array_equal(h1.view(np.int64), h2.view(np.int64))


def test_pcg_rejects_an_out_of_range_column(require_gpu):
    A = _csr(problems.laplacian_2d(6))
    M = _csr(problems.diagonal_inverse(A))
    bad = A.indices.astype(np.int64)
    bad[7] = A.shape[0] + 2
    with pytest.raises(RuntimeError, match="CSR column index out of range"):
        backward_error.pcg(A.data, bad, A.indptr, M.data, M.indices, M.indptr, np.ones(A.shape[0]), 50, 1, 1e-8)
    # the library stays usable
    hist, status = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr,
                                      np.ones(A.shape[0]), 50, 1, 1e-8)
    assert status == 1


def test_pcg_symmetric_part_with_a_row_longer_than_the_shared_memory_sort(require_gpu):
    """(M + M^T)/2 on the device when M has a dense column: its transpose has a
    row of n > 8,192 entries, which the transpose sorts by chunks and merge
    passes (three chunks here).  The device preconditioner must equal scipy's
    (M + M^T) * 0.5, so PCG with it matches PCG given scipy's result, bit for bit."""
    A = _csr(problems.laplacian_2d(142))
    n = A.shape[0]
    assert n > 2 * 8192
    rng = np.random.default_rng(6)
    dense_column = sparse.csr_matrix((1e-4 * rng.standard_normal(n), (np.arange(n), np.full(n, 7))), shape=(n, n))
    M = _csr(problems.diagonal_inverse(A) + dense_column)
    S = _csr((M + M.T) * 0.5)
    b, _ = problems.solution_rhs(A, seed=3)
    h1, s1 = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, b, 800, 1, 1e-8,
                                symmetric_part=True)
    h2, s2 = backward_error.pcg(A.data, A.indices, A.indptr, S.data, S.indices, S.indptr, b, 800, 1, 1e-8)
    assert s1 == s2
    assert np.array_equal(h1.view(np.int64), h2.view(np.int64))
