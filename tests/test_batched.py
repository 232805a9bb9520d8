"""Batched Global MR (spai_mr_batched): every system of a batch must come
out exactly as it does alone -- against the oracle per system in FP64, and
against single-system device runs in mixed precision -- with early stops at
different iterations.  The input checks run on the CPU."""
import ctypes

import numpy as np
import pytest
from scipy import sparse

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib, global_spai, problems
from parallellocallyoptimalapproximatesparsematrixinverses_b200.methods import as_csc, matrix_data
from tests.conftest import cuda_available
from tests.helpers import assert_same_result


def _mixed_sizes():
    return [problems.laplacian_2d(9), problems.diffusion_2d(12, 1.0, 1), problems.diffusion_3d(5, 1.0, 2),
            problems.tridiagonal(40), problems.random_banded_spd(3000, 2, 2, 3), problems.laplacian_2d(5)]


def _oracle(A, M0=None, **kw):
    return pyoracle.run("global_spai", "mr", A, M0=M0, order=pyoracle.ORDER_DEVICE, **kw)


# ---- CPU: input checks before any device work ------------------------------

def test_batched_needs_per_column_dropping():
    with pytest.raises(RuntimeError, match="topk_per_column > 0 or enable_dropping = 0"):
        global_spai.mr_batched([problems.laplacian_2d(4)], max_density=1.0)


def test_batched_rejects_an_explicit_preconditioner():
    lib = _lib.load()
    A = as_csc(problems.laplacian_2d(4))
    a = (_lib.MatrixData * 1)(matrix_data(A))
    params = _lib.MethodParams(5, 1e-8, 1.0, 0, 1, 0, 1, 2)
    results = (_lib.Result * 1)()
    err = ctypes.create_string_buffer(256)
    assert lib.spai_mr_batched(1, a, None, params, None, results, err, len(err)) == -1
    assert b"use_preconditioner must be 0" in err.value
    assert not results[0].col_offsets and not results[0].error_message


def test_batched_validates_every_system_with_the_reference_messages():
    # the second system's budget cannot hold its diagonal (methods_common.cpp:12-36)
    with pytest.raises(RuntimeError, match="too small to preserve the diagonal"):
        global_spai.mr_batched([problems.laplacian_2d(10), problems.tridiagonal(3)], max_density=0.05,
                               topk_per_column=3)
    with pytest.raises(ValueError, match="one matrix per system"):
        global_spai.mr_batched([problems.laplacian_2d(4)], M0s=[], topk_per_column=3)


@pytest.mark.skipif(cuda_available(), reason="checks the no-device error path")
def test_batched_fails_loudly_without_a_device():
    with pytest.raises(RuntimeError, match="no CUDA device"):
        global_spai.mr_batched([problems.laplacian_2d(4)], max_density=1.0, topk_per_column=3)


# ---- GPU -------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("topk", [3, 7])
def test_fp64_batched_matches_oracle_per_system(require_gpu, topk):
    systems = _mixed_sizes()
    kw = dict(max_iterations=8, tolerance=1e-10, max_density=1.0)
    got = global_spai.mr_batched(systems, topk_per_column=topk, **kw)
    assert len(got) == len(systems)
    for b, A in enumerate(systems):
        assert_same_result(got[b], _oracle(A, topk_per_column=topk, **kw), f"system {b} top-{topk}")


@pytest.mark.gpu
def test_fp64_batched_stops_each_system_on_its_own(require_gpu):
    systems = _mixed_sizes()
    # system 3 starts at its exact inverse (converged at iteration 0); with
    # ||R|| < 1 as the goal, systems 5, 0 and 2 converge at iterations 2, 6
    # and 7, and systems 1 and 4 run to the limit
    M0s = [problems.diagonal_inverse(A) for A in systems]
    M0s[3] = sparse.csc_matrix(np.linalg.inv(systems[3].toarray()))
    kw = dict(max_iterations=25, tolerance=1.0, max_density=1.0)
    got = global_spai.mr_batched(systems, M0s=M0s, topk_per_column=40, **kw)
    iterations = set()
    for b, A in enumerate(systems):
        want = _oracle(A, M0=M0s[b], topk_per_column=40, **kw)
        assert_same_result(got[b], want, f"system {b}")
        iterations.add(want.iterations)
    assert got[3].iterations == 0 and got[3].converged
    assert iterations == {0, 2, 6, 7, 25}


@pytest.mark.gpu
def test_fp64_batched_density_stop_without_dropping(require_gpu):
    systems = [problems.laplacian_2d(8), problems.diffusion_2d(10, 1.0, 4), problems.tridiagonal(60)]
    # the density limit 0.25 stops the systems at iterations 3, 4 and 8
    kw = dict(max_iterations=10, tolerance=1e-12, max_density=0.25, enable_dropping=False)
    got = global_spai.mr_batched(systems, **kw)
    for b, A in enumerate(systems):
        assert_same_result(got[b], _oracle(A, **kw), f"system {b}")
    assert [r.iterations for r in got] == [3, 4, 8]


@pytest.mark.gpu
def test_mixed_batched_matches_single_system_runs(require_gpu):
    systems = _mixed_sizes()
    kw = dict(max_iterations=6, tolerance=1e-10, max_density=1.0, topk_per_column=5, precision="mixed")
    got = global_spai.mr_batched(systems, **kw)
    for b, A in enumerate(systems):
        assert_same_result(got[b], global_spai.mr(A, **kw), f"mixed system {b}")


@pytest.mark.gpu
def test_fp64_diffusion_batch_matches_oracle(require_gpu):
    # the many-systems workload (log-uniform sizes, 2-D and 3-D, sigma 0.5, shifted), scaled down
    systems = problems.diffusion_batch(count=24, seed=3, n_min=500, n_max=8000)
    kw = dict(max_iterations=15, tolerance=1e-10, max_density=1.0)
    got = global_spai.mr_batched(systems, topk_per_column=10, **kw)
    for b, A in enumerate(systems):
        assert_same_result(got[b], _oracle(A, topk_per_column=10, **kw), f"system {b}")
