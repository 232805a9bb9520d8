"""The reference's own experiment drivers, unchanged, against this library.

oracle/build_drivers.sh compiles the reference's scripts/methods_convergence.py,
scripts/common.py and scripts/utils/{methods,typst,backward_error}.py with
Cython (no edits) into oracle/_ref/drivers/, beside the reference's ten sample
matrices and its recorded result CSVs (scripts/results/results_sample).  Here
`methods_convergence.main()` runs with `methods_cython` resolved to this
library's compat shims, so every SPAI build and every PCG solve in the
driver goes through libspai_b200.so; matplotlib, absent from this image, is
replaced by a do-nothing test double (tests/driver_stubs) because plotting is
not checked.

Each recorded run (dropping or not, iteration limit, density limit, matrix)
is replayed in one of two ways:

* full: the driver's own arguments (scripts/results/results_sample path
  names; 256 requested threads; backward error with 1 realization, seed 1,
  150 PCG iterations), and all four CSVs it writes compared with the
  recorded ones;
* prefix: the same arguments with a shorter iteration limit and no backward
  error, and the convergence rows written compared with the recorded ones --
  for the runs whose full length would take minutes on one GPU.

What is compared, and how:

* convergence.csv (the ||R||_F history of every method): as text, so bit for
  bit -- the library runs the reference's summation order;
* construction_status.csv: every field as text except the two the driver
  computes on the host with scipy from the returned M (`actual_residual_norm`,
  `construction_backward_error`), which agree to 1e-12 relative: the
  recording environment's scipy summed I - A M in another order;
* solver_status.csv and backward_error.csv (PCG on the saved M, through the
  library's PCG): the recording's dot products are OpenMP reductions over 256
  threads (backward_error.pyx:37-42), whose combining order OpenMP leaves
  open, so those last bits are not reproducible even by the reference; the
  library sums in its fixed tree.  The histories agree to rounding at first;
  later they drift, slowly for a symmetric M and by tens of updates for the
  non-symmetric M of Global MR, with which PCG is not a symmetric method.
  Compared are the labels and settings as text (method, realization, solver,
  threads, history limit) and the first 20 updates of every history within
  1e-6 relative (1e-12 absolute).
"""
import csv
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
DRIVERS = ROOT / "oracle" / "_ref" / "drivers"
SCRIPTS = DRIVERS / "scripts"
RECORDED = DRIVERS / "recorded"
STUBS = ROOT / "tests" / "driver_stubs"
COMPAT = ROOT / "parallellocallyoptimalapproximatesparsematrixinverses_b200" / "compat"

# (dropping, iteration limit, density limit, matrix) -> None (full) or the prefix length
RUNS = {
    ("dropping", 100, "0.030", "4bw100eigs20k2"): None,
    ("dropping", 100, "0.030", "Poisson32k"): 5,
    ("dropping", 100, "0.030", "wathen100"): 5,
    ("dropping", 1000, "0.030", "bcsstk21"): 100,
    ("dropping", 500, "0.030", "4bw100eigs20k"): 50,
    ("dropping", 500, "0.030", "bundle1"): 5,
    ("dropping", 500, "0.030", "rand20k"): 5,
    ("dropping", 500, "0.030", "rand20k2"): 3,
    ("dropping", 500, "0.030", "tri100eigs4k"): None,
    ("dropping", 5000, "0.030", "msc04515"): 100,
    ("no_dropping", 100, "0.030", "4bw100eigs20k2"): None,
    ("no_dropping", 100, "0.030", "Poisson32k"): 5,
    ("no_dropping", 100, "0.030", "rand20k"): 3,
    ("no_dropping", 100, "0.030", "wathen100"): 5,
    ("no_dropping", 1000, "1.000", "bcsstk21"): 30,
    ("no_dropping", 500, "0.030", "4bw100eigs20k"): 20,
    ("no_dropping", 500, "0.030", "bundle1"): 2,
    ("no_dropping", 500, "0.030", "rand20k2"): 3,
    ("no_dropping", 500, "1.000", "tri100eigs4k"): 30,
    ("no_dropping", 5000, "0.030", "msc04515"): None,
}


def _tag(mode, iterations, density):
    return f"{mode}-max_iter_{iterations}-max_density_{density}"


def _read(path):
    with open(path, newline="", encoding="utf-8") as f:
        return list(csv.reader(f))


def run_driver(mode, iterations, density, matrix, out_dir, backward_error=True, timeout=1800):
    """Runs the compiled reference driver; returns the directory it wrote."""
    args = ["--output-dir", str(out_dir), "--datasets", matrix, "--datasets-dir", str(SCRIPTS / "sample_datasets"),
            "--max-iterations", str(iterations), "--max-density", density, "--num-threads", "256"]
    if mode == "no_dropping":
        args.append("--disable-dropping")
    if not backward_error:
        args.append("--no-backward-error")
    code = f"import sys; sys.argv = ['methods_convergence'] + {args!r}; import methods_convergence; " \
           "methods_convergence.main()"
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([str(STUBS), str(COMPAT), str(SCRIPTS), str(ROOT)])
    proc = subprocess.run([sys.executable, "-c", code], cwd=str(out_dir), env=env, capture_output=True, text=True,
                          timeout=timeout)
    assert proc.returncode == 0, proc.stderr[-3000:]
    return Path(out_dir) / mode / f"max_iter_{iterations}" / f"max_density_{density}" / matrix


def recorded_dir(mode, iterations, density, matrix):
    return RECORDED / mode / f"max_iter_{iterations}" / f"max_density_{density}" / matrix


HOST_COMPUTED = {"actual_residual_norm", "construction_backward_error"}


def _close(got, want, rel, absolute=0.0):
    g, w = float(got), float(want)
    return abs(g - w) <= absolute + rel * abs(w)


def _compare_rows(name, got, want, check):
    """First difference between two CSVs (header row first), or None."""
    if got[0] != want[0]:
        return f"{name}: header {got[0]} != {want[0]}"
    if len(got) != len(want):
        return f"{name}: {len(got)} rows, recorded {len(want)}"
    for r in range(1, len(got)):
        for c, key in enumerate(got[0]):
            if not check(key, got[r][c], want[r][c]):
                return f"{name}: row {r} {key}: got {got[r][c]} want {want[r][c]}"
    return None


def _construction_check(key, g, w):
    if key in HOST_COMPUTED:
        return _close(g, w, 1e-12)
    return g == w


PCG_OUTCOME = {"solver_updates", "final_relative_residual", "converged", "status"}


def _solver_check(key, g, w):
    # the outcome of a run depends on the reduction order (module docstring); the setting columns do not
    return key in PCG_OUTCOME or g == w


BACKWARD_ROWS = 20  # leading PCG updates compared value by value


def _backward_rows(name, got, want):
    """PCG histories: the same methods; lengths within one update; the first
    BACKWARD_ROWS updates equal to rounding (the final values are checked in
    solver_status.csv)."""
    if got[0] != want[0]:
        return f"{name}: header {got[0]} != {want[0]}"
    if abs(len(got) - len(want)) > 1:
        return f"{name}: {len(got)} rows, recorded {len(want)}"
    for r in range(1, min(len(got), len(want), BACKWARD_ROWS + 1)):
        for c in range(1, len(got[0])):
            g, w = got[r][c], want[r][c]
            if g == "" or w == "":
                continue  # one history ended a row earlier
            if not _close(g, w, 1e-6, 1e-12):
                return f"{name}: row {r} {got[0][c]}: got {g} want {w}"
    return None


def compare_full(got_dir, want_dir, mode, iterations, density):
    """Every CSV the recorded run left, compared as the module docstring says (empty list: all agree)."""
    tag = _tag(mode, iterations, density)
    checks = [
        (f"all-{tag}-convergence.csv", lambda n, g, w: _compare_rows(n, g, w, lambda k, a, b: a == b)),
        (f"all-{tag}-construction_status.csv", lambda n, g, w: _compare_rows(n, g, w, _construction_check)),
        (f"all-{tag}-max_backward_iter_150-solver_status.csv", lambda n, g, w: _compare_rows(n, g, w, _solver_check)),
        (f"all-{tag}-max_backward_iter_150-backward_error.csv", _backward_rows),
    ]
    problems = []
    for name, check in checks:
        want_path = want_dir / name
        if not want_path.exists():
            continue
        got_path = got_dir / name
        if not got_path.exists():
            problems.append(f"{name}: not written")
            continue
        problem = check(name, _read(got_path), _read(want_path))
        if problem:
            problems.append(problem)
    return problems


def compare_prefix(got_dir, want_dir, mode, iterations, density, prefix):
    got = _read(got_dir / f"all-{_tag(mode, prefix, density)}-convergence.csv")
    want = _read(want_dir / f"all-{_tag(mode, iterations, density)}-convergence.csv")
    problems = []
    if got[0] != want[0]:
        problems.append(f"header: got {got[0]} want {want[0]}")
    for r in range(1, len(got)):
        # a method that stopped before the prefix leaves '' in later rows, as recorded
        if got[r] != want[r]:
            problems.append(f"row {r}: got {got[r]} want {want[r]}")
            break
    return problems


@pytest.mark.gpu
@pytest.mark.parametrize("run", sorted(RUNS), ids=lambda r: f"{r[0]}-{r[1]}-{r[2]}-{r[3]}")
def test_reference_driver_replays_the_recorded_results(require_gpu, tmp_path, run):
    if not (SCRIPTS / "methods_convergence.py").exists() and not list(SCRIPTS.glob("methods_convergence*.so")):
        pytest.fail("oracle/_ref/drivers is not built: run oracle/build_drivers.sh where the reference tree is "
                    "present (build() does) before the GPU tests")
    mode, iterations, density, matrix = run
    prefix = RUNS[run]
    want_dir = recorded_dir(mode, iterations, density, matrix)
    if prefix is None:
        got_dir = run_driver(mode, iterations, density, matrix, tmp_path)
        problems = compare_full(got_dir, want_dir, mode, iterations, density)
    else:
        got_dir = run_driver(mode, prefix, density, matrix, tmp_path, backward_error=False)
        problems = compare_prefix(got_dir, want_dir, mode, iterations, density, prefix)
    assert not problems, "\n".join(problems)
