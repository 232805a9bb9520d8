"""Compiled callers of the boundary: a C++ program written against the C++ API
(include/methods.hpp, the reference's include/methods.hpp names over the
C ABI) and a C99 program written against include/spai_b200.h, both linked
against libspai_b200.so.

Without a GPU the programs must compile, link and resolve every symbol; on a
GPU the C++ program runs the reference's own C++ test properties
(reference tests/test.cpp:107-179) and its results are compared bit for bit
with the oracle in the reference's summation order."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest
from scipy import sparse

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "parallellocallyoptimalapproximatesparsematrixinverses_b200"
BUILD = PKG / "_build"


def _build(source: str, compiler: list, out_name: str) -> Path:
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import _lib
    _lib.load()  # builds libspai_b200.so when it is missing
    BUILD.mkdir(exist_ok=True)
    out = BUILD / out_name
    cmd = [*compiler, "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / source), "-L", str(PKG),
           "-lspai_b200", f"-Wl,-rpath,{PKG}", "-o", str(out)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    return out


def _cxx():
    return _build("methods_api_test.cpp", ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror"],
                  "methods_api_test")


def _c():
    return _build("c_abi_caller.c", ["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror"], "c_abi_caller")


def _symbols(path: Path) -> set:
    out = subprocess.run(["nm", "-D", "--undefined-only", str(path)], capture_output=True, text=True, check=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}


def test_cpp_api_and_c_caller_compile_and_link():
    cxx = _cxx()
    c = _c()
    # the C++ API is header-only: the program binds the reference's C entry points themselves
    needed = _symbols(cxx)
    for name in ("spai_global_cg", "spai_global_mr", "spai_global_lomr", "inner_outer_mr", "inner_outer_lomr",
                 "free_mem"):
        assert name in needed, name
    assert {"spai_run_ex", "free_mem"} <= _symbols(c)
    # every symbol resolves against the library (the dynamic loader would refuse otherwise)
    proc = subprocess.run(["ldd", "-r", str(cxx)], capture_output=True, text=True)
    assert "undefined symbol" not in proc.stdout + proc.stderr


def _oracle_runs():
    from oracle import pyoracle
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import problems
    A = problems.tridiagonal(12)
    eye = sparse.identity(12, format="csc")
    runs = {}
    for family, name, label in (("global_spai", "cg", "global_cg"), ("global_spai", "mr", "global_mr"),
                                ("global_spai", "lomr", "global_lomr"), ("inner_outer", "mr", "inner_outer_mr"),
                                ("inner_outer", "lomr", "inner_outer_lomr")):
        runs[label + "_p1"] = pyoracle.run(family, name, A, M0=eye, Pr=eye, max_iterations=8, tolerance=1e-14,
                                           max_density=1.0, num_threads=1, order=pyoracle.ORDER_REFERENCE)
        runs[label + "_drop"] = pyoracle.run(family, name, A, M0=eye, Pr=eye, max_iterations=3, tolerance=0.0,
                                             max_density=0.12, num_threads=1, order=pyoracle.ORDER_REFERENCE)
    return runs


@pytest.mark.gpu
def test_cpp_api_runs_the_reference_checks_and_matches_the_oracle(require_gpu):
    exe = _cxx()
    proc = subprocess.run([str(exe), "--dump"], capture_output=True, text=True, timeout=600,
                          env=dict(os.environ))
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "all checks passed" in proc.stdout
    want = _oracle_runs()
    seen = 0
    for line in proc.stdout.splitlines():
        parts = line.split()
        if not parts or parts[0] not in want:
            continue
        bar = parts.index("|")
        iterations = int(parts[1])
        residuals = np.array([float(v) for v in parts[2:bar]])
        values = np.array([float(v) for v in parts[bar + 2:]])
        w = want[parts[0]]
        assert iterations == w.iterations, parts[0]
        assert np.array_equal(residuals.view(np.int64), w.history["residual_norm"].view(np.int64)), parts[0]
        assert np.array_equal(values.view(np.int64), sparse.csc_matrix(w.M).data.view(np.int64)), parts[0]
        seen += 1
    assert seen == len(want)


@pytest.mark.gpu
def test_c_caller_runs(require_gpu):
    exe = _c()
    proc = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert proc.stdout.startswith("iterations 10 ")
