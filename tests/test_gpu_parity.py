"""GPU (FP64) results through the C ABI against the CPU oracle in the
device summation order: M pattern, M values and the whole iteration history
must be bit-identical.  The oracle itself is pinned to the reference's
recorded outputs by tests/test_oracle_golden.py."""
import numpy as np
import pytest

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import global_spai, inner_outer, problems
from tests.helpers import METHODS, assert_same_result

pytestmark = pytest.mark.gpu

FAMILIES = {"global_spai": global_spai, "inner_outer": inner_outer}


def _run_both(family, name, A, M0, Pr, topk=0, **kw):
    method = getattr(FAMILIES[family], name)
    ext = {"topk_per_column": topk} if topk else {}
    got = method(A, M0=M0, Pr=Pr, **kw, **ext)
    want = pyoracle.run(family, name, A, M0=M0, Pr=Pr, order=pyoracle.ORDER_DEVICE, topk_per_column=topk, **kw)
    return got, want


CASES = {
    # reference tests/test.cpp:111 fixture: tridiag n=12, M0 = Pr = I, 8 iterations, tol 1e-14, density 1
    "tridiag_dense": dict(maker=lambda: problems.tridiagonal(12), identity=True,
                          kw=dict(max_iterations=8, tolerance=1e-14, max_density=1.0)),
    # tests/test.cpp:141-151: dropping to density 0.12, 3 iterations
    "tridiag_drop": dict(maker=lambda: problems.tridiagonal(12), identity=True,
                         kw=dict(max_iterations=3, tolerance=0.0, max_density=0.12)),
    # tests/test.cpp:153-165: no dropping, density stop 0.2
    "tridiag_nodrop": dict(maker=lambda: problems.tridiagonal(12), identity=True,
                           kw=dict(max_iterations=8, tolerance=0.0, max_density=0.2, enable_dropping=False)),
    # 5-point Laplacian 16x16 with the global budget active
    "lap16_budget": dict(maker=lambda: problems.laplacian_2d(16), identity=False,
                         kw=dict(max_iterations=10, tolerance=1e-12, max_density=0.02)),
    # variable-coefficient 2-D diffusion, no dropping
    "diff12_nodrop": dict(maker=lambda: problems.diffusion_2d(12, 1.0, 3), identity=False,
                          kw=dict(max_iterations=6, tolerance=1e-12, max_density=1.0, enable_dropping=False)),
}


@pytest.mark.parametrize("family,name", METHODS)
@pytest.mark.parametrize("case", sorted(CASES))
def test_fp64_matches_oracle(require_gpu, family, name, case):
    spec = CASES[case]
    A = spec["maker"]()
    n = A.shape[0]
    if spec["identity"]:
        from scipy import sparse
        M0 = sparse.identity(n, format="csc")
        Pr = sparse.identity(n, format="csc")
    else:
        M0 = problems.diagonal_inverse(A)
        Pr = None
    got, want = _run_both(family, name, A, M0, Pr, **spec["kw"])
    assert_same_result(got, want, f"{family}.{name} {case}")


@pytest.mark.parametrize("family,name", METHODS)
def test_fp64_topk_matches_oracle(require_gpu, family, name):
    A = problems.laplacian_2d(16)
    M0 = problems.diagonal_inverse(A)
    got, want = _run_both(family, name, A, M0, None, topk=5, max_iterations=8, tolerance=1e-12, max_density=0.05)
    assert_same_result(got, want, f"{family}.{name} top-5")
    assert np.diff(got.M.indptr).max() <= 5
