"""The oracle PCG against the reference's own PCG (compiled from
methods_cython/backward_error.pyx): bit-identical in the reference's
sequential order; same status and +-1 iteration in the device order."""
from pathlib import Path

import numpy as np
import pytest
from scipy import sparse

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import problems

GOLDEN = Path(__file__).resolve().parent / "golden"


def _tri4k():
    z = np.load(GOLDEN / "tri100eigs4k.npz")
    return sparse.csc_matrix((z["data"], z["indices"], z["indptr"]), shape=tuple(z["shape"]))


CASES = {
    "diff2d_24_jacobi": lambda: problems.diffusion_2d(24, 1.0, 5),
    "lap2d_32_jacobi": lambda: problems.laplacian_2d(32),
    "tri4k_jacobi": _tri4k,
}


@pytest.mark.parametrize("label", sorted(CASES))
@pytest.mark.parametrize("tol", [1e-6, 1e-8])
def test_oracle_pcg_matches_reference(label, tol):
    gold = np.load(GOLDEN / "pcg_reference.npz")
    want = gold[f"{label}_tol{tol:g}_history"]
    want_status = int(gold[f"{label}_tol{tol:g}_status"])
    A = sparse.csr_matrix(CASES[label]())
    A.sort_indices()
    M = sparse.csr_matrix(problems.diagonal_inverse(A))
    b, _ = problems.solution_rhs(A, seed=0)
    got, status = pyoracle.pcg(A, M, b, 3000, tol, order=pyoracle.ORDER_REFERENCE)
    assert status == want_status
    assert np.array_equal(got.view(np.int64), want.view(np.int64))
    dev, dev_status = pyoracle.pcg(A, M, b, 3000, tol, order=pyoracle.ORDER_DEVICE)
    assert dev_status == want_status
    assert abs(len(dev) - len(want)) <= 1


def test_pcg_status_codes():
    A = sparse.csr_matrix(problems.laplacian_2d(8))
    M = sparse.csr_matrix(problems.diagonal_inverse(A))
    b, _ = problems.solution_rhs(A, seed=1)
    hist, status = pyoracle.pcg(A, M, b, 3, 1e-12)
    assert status == 0 and len(hist) == 3 and hist[0] == 1.0
    # zero preconditioner: r.z = 0 -> recurrence breakdown (status 2)
    Z = sparse.csr_matrix(A.shape)
    hist, status = pyoracle.pcg(A, Z, b, 10, 1e-12)
    assert status == 2
