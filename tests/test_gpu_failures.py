"""Failure paths on the device, with the failures made on the host: an
allocation that fails part-way through a call (spai_inject_allocation_failure)
is reported through the usual error path and leaves the library usable, and
a bad diagonal is refused with the reference's message (methods_common.cpp:50-63)."""
import numpy as np
import pytest
from scipy import sparse

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib, backward_error, global_spai, problems
from tests.helpers import assert_same_result

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("after", [8, 30, 90])
def test_allocation_failure_is_reported_and_the_library_recovers(require_gpu, after):
    lib = _lib.load()
    A = problems.diffusion_2d(23, 1.0, 9)
    M0 = problems.diagonal_inverse(A)
    kw = dict(max_iterations=6, tolerance=1e-12, max_density=0.05)
    lib.spai_inject_allocation_failure(after)
    try:
        with pytest.raises(RuntimeError, match="injected allocation failure"):
            global_spai.mr(A, M0=M0, **kw)
    finally:
        lib.spai_inject_allocation_failure(-1)
    got = global_spai.mr(A, M0=M0, **kw)
    # a call with only the reference's arguments runs in the reference's summation order
    want = pyoracle.run("global_spai", "mr", A, M0=M0, order=pyoracle.ORDER_REFERENCE, **kw)
    assert_same_result(got, want, f"after an injected failure at reservation {after}")


def test_allocation_failure_in_pcg(require_gpu):
    lib = _lib.load()
    A = sparse.csr_matrix(problems.diffusion_2d(21, 1.0, 2))
    A.sort_indices()
    M = sparse.csr_matrix(problems.diagonal_inverse(A))
    b, _ = problems.solution_rhs(A, seed=3)
    lib.spai_inject_allocation_failure(4)
    try:
        with pytest.raises(RuntimeError, match="injected allocation failure"):
            backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, b, 500, 1, 1e-8)
    finally:
        lib.spai_inject_allocation_failure(-1)
    hist, status = backward_error.pcg(A.data, A.indices, A.indptr, M.data, M.indices, M.indptr, b, 500, 1, 1e-8)
    want, want_status = pyoracle.pcg(A, M, b, 500, 1e-8, order=pyoracle.ORDER_DEVICE)
    assert status == want_status == 1 and np.array_equal(hist.view(np.int64), want.view(np.int64))


@pytest.mark.parametrize("diagonal", [0.0, -1.0])
def test_bad_diagonal_is_refused_with_the_reference_message(require_gpu, diagonal):
    A = sparse.lil_matrix(problems.laplacian_2d(5))
    A[3, 3] = diagonal
    A = sparse.csc_matrix(A)
    with pytest.raises(RuntimeError, match="A has an invalid diagonal entry; provide Pr explicitly"):
        global_spai.mr(A, max_density=1.0)
    # with Pr given, the diagonal is not needed
    r = global_spai.mr(A, Pr=sparse.identity(25, format="csc"), max_iterations=2, max_density=1.0)
    assert r.iterations >= 1
