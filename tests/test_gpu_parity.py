"""GPU (FP64) results through the C ABI against the CPU oracle in the
device summation order: M pattern, M values and the whole iteration history
must be bit-identical.  The oracle itself is pinned to the reference's
recorded outputs by tests/test_oracle_golden.py."""
import numpy as np
import pytest

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import global_spai, inner_outer, problems
from tests.helpers import METHODS, assert_same_result, relative_difference

pytestmark = pytest.mark.gpu

FAMILIES = {"global_spai": global_spai, "inner_outer": inner_outer}


def _run_both(family, name, A, M0, Pr, topk=0, **kw):
    method = getattr(FAMILIES[family], name)
    ext = {"topk_per_column": topk} if topk else {}
    got = method(A, M0=M0, Pr=Pr, summation="device", **kw, **ext)
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


@pytest.mark.parametrize("family,name", [("global_spai", "mr"), ("global_spai", "cg"), ("inner_outer", "lomr")])
@pytest.mark.parametrize("topk", [0, 6])
def test_fp64_wide_windows_hash_path(require_gpu, family, name, topk):
    # random long-range couplings: row windows wider than the bitmap kernels take
    A = problems.random_banded_spd(70_000, half_width=2, extra=2, seed=4)
    M0 = problems.diagonal_inverse(A)
    got, want = _run_both(family, name, A, M0, None, topk=topk, max_iterations=2, tolerance=1e-12,
                          max_density=6.0 / A.shape[0])
    assert_same_result(got, want, f"{family}.{name} wide top-{topk}")


def _arrow(n):
    """SPD arrow matrix: a dense first row and column over a diagonal."""
    from scipy import sparse
    rng = np.random.default_rng(11)
    off = rng.uniform(0.1, 1.0, n - 1) / np.sqrt(n)
    rows = np.concatenate([np.arange(1, n), np.zeros(n - 1, dtype=np.int64), np.arange(n)])
    cols = np.concatenate([np.zeros(n - 1, dtype=np.int64), np.arange(1, n), np.arange(n)])
    vals = np.concatenate([off, off, np.full(n, 4.0)])
    a = sparse.csc_matrix((vals, (rows, cols)), shape=(n, n))
    a.sort_indices()
    return a


@pytest.mark.parametrize("family,name", METHODS)
def test_fp64_long_columns_fallbacks(require_gpu, family, name):
    # a column of n entries: longer than the fused drop kernel and the warp union take
    A = _arrow(1500)
    M0 = problems.diagonal_inverse(A)
    got, want = _run_both(family, name, A, M0, None, max_iterations=3, tolerance=1e-14, max_density=0.5)
    assert_same_result(got, want, f"{family}.{name} arrow")


@pytest.mark.parametrize("family,name", METHODS)
@pytest.mark.parametrize("topk", [0, 8])
def test_mixed_precision_error_against_fp64_oracle(require_gpu, family, name, topk):
    """FP32 storage of A, M, R, Z with FP64 reductions, against the FP64 oracle:
    ||R||_F histories within 1e-4 relative at every iteration and
    ||M_mixed - M_fp64||_F / ||M_fp64||_F within 1e-4 (f32 unit roundoff is 6e-8)."""
    A = problems.diffusion_2d(32, 1.0, 7)
    M0 = problems.diagonal_inverse(A)
    kw = dict(max_iterations=10, tolerance=1e-12, max_density=8.0 / A.shape[0])
    method = getattr(FAMILIES[family], name)
    ext = {"topk_per_column": topk} if topk else {}
    got = method(A, M0=M0, precision="mixed", **kw, **ext)
    want = pyoracle.run(family, name, A, M0=M0, order=pyoracle.ORDER_DEVICE, topk_per_column=topk, **kw)
    gh = got.history["residual_norm"]
    wh = want.history["residual_norm"]
    assert gh.shape == wh.shape
    hist_err = float(np.max(np.abs(gh - wh) / wh))
    m_err = relative_difference(got.M, want.M)
    assert hist_err <= 1e-4, f"{family}.{name} top-{topk}: history rel error {hist_err:.3e}"
    assert m_err <= 1e-4, f"{family}.{name} top-{topk}: M rel error {m_err:.3e}"


@pytest.mark.parametrize("topk", [0, 10])
def test_fp64_reference_cpu_configuration(require_gpu, topk):
    """The reference's own CPU-runnable case: 5-point Laplacian 64 x 64 (n = 4096),
    M0 = diag(A)^-1, Global MR for 20 iterations with dropping to 10 entries per
    column (global budget max_density = 10/n, or per-column top-10), then PCG
    to 1e-8 with the symmetric part of M on b = A x*, x* ~ N(0, 1) (seed 0)."""
    from scipy import sparse
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import backward_error
    A = problems.laplacian_2d(64)
    n = A.shape[0]
    M0 = problems.diagonal_inverse(A)
    got, want = _run_both("global_spai", "mr", A, M0, None, topk=topk, max_iterations=20, tolerance=1e-12,
                          max_density=10.0 / n)
    assert_same_result(got, want, f"laplacian 64x64 top-{topk}")
    msym = sparse.csr_matrix((got.M + got.M.T) * 0.5)
    msym.sort_indices()
    a = sparse.csr_matrix(A)
    a.sort_indices()
    b, _ = problems.solution_rhs(A, seed=0)
    hist, status = backward_error.pcg(a.data, a.indices, a.indptr, msym.data, msym.indices, msym.indptr, b, 2000, 1,
                                      1e-8)
    want_hist, want_status = pyoracle.pcg(a, msym, b, 2000, 1e-8, order=pyoracle.ORDER_DEVICE)
    assert status == want_status == 1
    assert np.array_equal(hist.view(np.int64), want_hist.view(np.int64))


@pytest.mark.parametrize("family,name", [("global_spai", "mr"), ("inner_outer", "lomr")])
def test_fp64_dense_column_global_hash_fallback(require_gpu, family, name):
    """A column with far more candidate rows than the shared-memory hash bins
    hold (about 630,000) over a window of 70,000 rows: the generic SpGEMM's
    hash in global memory, the two-pass union and no dropping (so the dense
    column survives every step)."""
    from scipy import sparse
    n = 70_000
    A = problems.random_banded_spd(n, half_width=2, extra=2, seed=6)
    dense = np.random.default_rng(12).uniform(-1.0, 1.0, n) * 1e-4
    M0 = sparse.lil_matrix(problems.diagonal_inverse(A))
    M0[:, 0] = dense[:, None]
    M0 = sparse.csc_matrix(M0)
    M0.sort_indices()
    got, want = _run_both(family, name, A, M0, None, max_iterations=2, tolerance=1e-12, max_density=1.0,
                          enable_dropping=False)
    assert_same_result(got, want, f"{family}.{name} dense column")


FUSED_CASES = {
    # 3-D 7-point, top-8: windows of several planes
    "diffusion_3d_16_top8": (lambda: problems.diffusion_3d(16, 1.0, 5), 8, 12),
    # 2-D 5-point, top-10, the reference's CPU-runnable shape
    "laplacian_64_top10": (lambda: problems.laplacian_2d(64), 10, 20),
    # a larger 3-D problem with the bench's top-16, a few iterations
    "diffusion_3d_40_top16": (lambda: problems.diffusion_3d(40, 1.0, 2), 16, 6),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", sorted(FUSED_CASES))
def test_fused_graph_mr_matches_unfused_kernels(require_gpu, case, precision):
    """Global MR with per-column top-k runs its iterations as one CUDA graph of
    fused kernels (mr_fused.cu); switched off, the same run goes through the
    unfused kernels.  Both must give the same bits: M and the whole history."""
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib
    maker, topk, iterations = FUSED_CASES[case]
    A = maker()
    n = A.shape[0]
    kw = dict(M0=problems.diagonal_inverse(A), max_iterations=iterations, tolerance=1e-12,
              max_density=topk / n, topk_per_column=topk, precision=precision, summation="device")
    lib = _lib.load()
    lib.spai_set_fused_mr(0)
    try:
        want = global_spai.mr(A, **kw)
    finally:
        lib.spai_set_fused_mr(1)
    got = global_spai.mr(A, **kw)
    assert_same_result(got, want, f"{case} {precision}")
    if precision == "fp64":
        oracle = pyoracle.run("global_spai", "mr", A, M0=kw["M0"], max_iterations=iterations, tolerance=1e-12,
                              max_density=topk / n, topk_per_column=topk, order=pyoracle.ORDER_DEVICE)
        assert_same_result(got, oracle, f"{case} against the oracle")


def test_fused_graph_mr_profiled_steps_match(require_gpu):
    """With the library's event accounting on, the fused kernels run one launch
    at a time (no graph); the results are the same bits."""
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib
    A = problems.diffusion_3d(16, 1.0, 5)
    n = A.shape[0]
    kw = dict(M0=problems.diagonal_inverse(A), max_iterations=8, tolerance=1e-12, max_density=8 / n,
              topk_per_column=8, precision="mixed")
    lib = _lib.load()
    want = global_spai.mr(A, **kw)
    lib.spai_profile_reset()
    lib.spai_profile_enable(1)
    try:
        got = global_spai.mr(A, **kw)
    finally:
        lib.spai_profile_enable(0)
    assert_same_result(got, want, "profiled fused steps")
