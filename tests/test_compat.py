"""The methods_cython shims: with the compat directory on sys.path, the
imports the reference's drivers make (scripts/utils/methods.py:3,
scripts/utils/backward_error.py:9) resolve to this library."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
COMPAT = ROOT / "parallellocallyoptimalapproximatesparsematrixinverses_b200" / "compat"

PROBE = r"""
import inspect
from methods_cython import global_spai, inner_outer, OutputResult
from methods_cython.backward_error import matvec, pcg, parallel_threads
import parallellocallyoptimalapproximatesparsematrixinverses_b200 as pkg
assert global_spai is pkg.global_spai and inner_outer is pkg.inner_outer
assert pcg is pkg.pcg and matvec is pkg.matvec
assert global_spai.available_methods == ("cg", "mr", "lomr") and inner_outer.available_methods == ("mr", "lomr")
sig = inspect.signature(global_spai.mr)
assert list(sig.parameters)[:8] == ["A", "M0", "Pr", "max_iterations", "tolerance", "max_density",
                                    "enable_dropping", "num_threads"], list(sig.parameters)
assert list(inspect.signature(inner_outer.lomr).parameters)[8] == "inner_iterations"
assert list(inspect.signature(pcg).parameters)[:10] == ["a_values", "a_indices", "a_offsets", "m_values",
                                                        "m_indices", "m_offsets", "b", "max_iterations",
                                                        "threads", "tolerance"]
assert parallel_threads(5, 3) == 3 and parallel_threads(2, 9) == 2
print("ok")
"""


def test_methods_cython_shims_resolve_to_this_library():
    env = dict(os.environ, PYTHONPATH=os.pathsep.join([str(COMPAT), str(ROOT)]))
    out = subprocess.run([sys.executable, "-c", PROBE], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"


def test_parallel_threads_rejects_like_the_reference():
    from parallellocallyoptimalapproximatesparsematrixinverses_b200.compat.methods_cython.backward_error import (
        parallel_threads)
    with pytest.raises(ValueError):
        parallel_threads(0, 1)


DRIVERS = ROOT / "oracle" / "_ref" / "drivers" / "scripts"
DRIVER_PROBE = r"""
import common, methods_convergence
import scripts.utils.backward_error as be
import parallellocallyoptimalapproximatesparsematrixinverses_b200 as pkg
assert common.methods.global_spai is pkg.global_spai and common.methods.inner_outer is pkg.inner_outer
assert be.pcg is pkg.pcg and be.matvec is pkg.matvec
assert len(common.SAMPLE_DATASETS) == 10
print("ok")
"""


def test_compiled_reference_drivers_bind_to_this_library():
    """The reference's drivers, compiled unchanged by oracle/build_drivers.sh,
    import and reach this library through the shims (no GPU call is made)."""
    if not list(DRIVERS.glob("methods_convergence*.so")):
        pytest.skip("oracle/_ref/drivers is built by build() where the reference tree is present")
    stubs = ROOT / "tests" / "driver_stubs"
    env = dict(os.environ, PYTHONPATH=os.pathsep.join([str(stubs), str(COMPAT), str(DRIVERS), str(ROOT)]))
    out = subprocess.run([sys.executable, "-c", DRIVER_PROBE], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "ok"
