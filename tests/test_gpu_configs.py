"""The benchmark configurations beyond the headline one, on the GPU:

* 64^3 7-point log-normal diffusion (sigma 1), Global CG and LOMR with
  top-16, 30 iterations: FP64 bit for bit against the oracle (device order)
  on the 32^3 operator of the same generator, and at 64^3 the mixed-precision
  error against the FP64 device run stated and bounded, with PCG (FP32
  M-apply, refresh every 50) needing the same number of iterations.
* Inner-Outer LOMR on the random banded SPD matrix (band 4, 6 random
  off-diagonals per row, diagonal 1.05 x row sum), 5 outer x 10 inner, top-12:
  FP64 bit for bit against the oracle at n = 2^11, and the mixed error at
  n = 2^14.  n = 2^20 does not fit one GPU: the inner products Z = M_outer R
  and A Z are not dropped (inner_outer_common.hpp:41-42), and with random
  long-range couplings A Z holds tens of thousands of entries per column
  after the first outer iteration -- about 10^10 entries at n = 2^20 -- which
  the whole-matrix products cannot hold in 180 GB.

The oracle itself is pinned to the reference's recorded runs
(tests/test_oracle_golden.py)."""
import os

import numpy as np
import pytest
from scipy import sparse

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import backward_error, global_spai, inner_outer, problems
from tests.helpers import assert_same_result, relative_difference

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _mixed_error(mixed, fp64):
    gh = mixed.history["residual_norm"]
    wh = fp64.history["residual_norm"]
    assert gh.shape == wh.shape
    return float(np.max(np.abs(gh - wh) / wh)), relative_difference(mixed.M, fp64.M)


def _pcg_iterations(A, M, b, m_precision):
    a = sparse.csr_matrix(A)
    a.sort_indices()
    h, status = backward_error.pcg(a.data, a.indices, a.indptr, M.data, M.indices, M.indptr, b, 5000, 1, 1e-8,
                                   refresh_period=50, m_precision=m_precision, symmetric_part=True)
    assert status == 1
    return len(h) - 1


@pytest.mark.parametrize("name", ["cg", "lomr"])
def test_diffusion_3d_cg_lomr_fp64_matches_the_oracle(require_gpu, name):
    A = problems.diffusion_3d(32, 1.0, 0)
    n = A.shape[0]
    kw = dict(M0=problems.diagonal_inverse(A), max_iterations=30, tolerance=1e-12, max_density=16.0 / n,
              topk_per_column=16)
    got = getattr(global_spai, name)(A, precision="fp64", **kw)
    want = pyoracle.run("global_spai", name, A, order=pyoracle.ORDER_DEVICE, omp_threads=THREADS, **kw)
    assert_same_result(got, want, f"global {name} 32^3 top-16")


@pytest.mark.parametrize("name", ["cg", "lomr", "mr"])
def test_diffusion_3d_64_mixed_error_against_fp64(require_gpu, name):
    """Measured on a B200: ||M_mixed - M_fp64||_F / ||M_fp64||_F = 1.4e-4 (CG),
    8e-8 (LOMR), 2.2e-4 (MR); the residual histories agree within 2.3e-6
    relative; PCG takes 84, 80 and 80 iterations with either M."""
    A = problems.diffusion_3d(64, 1.0, 0)
    n = A.shape[0]
    kw = dict(M0=problems.diagonal_inverse(A), max_iterations=30, tolerance=1e-12, max_density=16.0 / n,
              topk_per_column=16)
    fp64 = getattr(global_spai, name)(A, precision="fp64", **kw)
    mixed = getattr(global_spai, name)(A, precision="mixed", **kw)
    hist_err, m_err = _mixed_error(mixed, fp64)
    assert hist_err <= 1e-5, f"{name}: history rel error {hist_err:.3e}"
    assert m_err <= 1e-3, f"{name}: M rel error {m_err:.3e}"
    b, _ = problems.solution_rhs(A, seed=0)
    its_fp64 = _pcg_iterations(A, fp64.M, b, "fp64")
    its_mixed = _pcg_iterations(A, mixed.M, b, "mixed")
    assert abs(its_fp64 - its_mixed) <= 1, (its_fp64, its_mixed)


def test_banded_inner_outer_lomr_fp64_matches_the_oracle(require_gpu):
    A = problems.random_banded_spd(1 << 11, half_width=4, extra=6, seed=0)
    n = A.shape[0]
    kw = dict(max_iterations=50, inner_iterations=10, tolerance=1e-12, max_density=12.0 / n, topk_per_column=12)
    got = inner_outer.lomr(A, precision="fp64", summation="device", **kw)
    want = pyoracle.run("inner_outer", "lomr", A, order=pyoracle.ORDER_DEVICE, omp_threads=THREADS, **kw)
    assert_same_result(got, want, "inner-outer lomr banded 2^11")


def test_banded_inner_outer_lomr_mixed_error(require_gpu):
    """Measured on a B200 at n = 2^14: history within 4.5e-9 relative and
    ||M_mixed - M_fp64||_F / ||M_fp64||_F = 1.2e-7, both over 50 iterations;
    the FP64 run is bit for bit the oracle's (device order)."""
    A = problems.random_banded_spd(1 << 14, half_width=4, extra=6, seed=0)
    n = A.shape[0]
    kw = dict(max_iterations=50, inner_iterations=10, tolerance=1e-12, max_density=12.0 / n, topk_per_column=12)
    fp64 = inner_outer.lomr(A, precision="fp64", summation="device", **kw)
    mixed = inner_outer.lomr(A, precision="mixed", **kw)
    assert fp64.iterations == mixed.iterations == 50
    hist_err, m_err = _mixed_error(mixed, fp64)
    assert fp64.history["residual_norm"][-1] < fp64.history["residual_norm"][0]
    assert hist_err <= 1e-6, f"history rel error {hist_err:.3e}"
    assert m_err <= 1e-5, f"M rel error {m_err:.3e}"
