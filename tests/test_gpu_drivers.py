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
  150 PCG iterations), and its convergence, construction-status,
  solver-status and backward-error CSVs compared with the recorded ones,
  field by field, as the text the driver writes (so floats bit for bit);
* prefix: the same arguments with a shorter iteration limit and no backward
  error, and the rows written compared with the recorded convergence rows --
  for the runs whose full length would take minutes on one GPU.
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
    ("dropping", 100, "0.030", "Poisson32k"): 8,
    ("dropping", 100, "0.030", "wathen100"): 8,
    ("dropping", 1000, "0.030", "bcsstk21"): None,
    ("dropping", 500, "0.030", "4bw100eigs20k"): 20,
    ("dropping", 500, "0.030", "bundle1"): 8,
    ("dropping", 500, "0.030", "rand20k"): None,
    ("dropping", 500, "0.030", "rand20k2"): 20,
    ("dropping", 500, "0.030", "tri100eigs4k"): None,
    ("dropping", 5000, "0.030", "msc04515"): 40,
    ("no_dropping", 100, "0.030", "4bw100eigs20k2"): None,
    ("no_dropping", 100, "0.030", "Poisson32k"): None,
    ("no_dropping", 100, "0.030", "rand20k"): None,
    ("no_dropping", 100, "0.030", "wathen100"): None,
    ("no_dropping", 1000, "1.000", "bcsstk21"): 20,
    ("no_dropping", 500, "0.030", "4bw100eigs20k"): 20,
    ("no_dropping", 500, "0.030", "bundle1"): None,
    ("no_dropping", 500, "0.030", "rand20k2"): None,
    ("no_dropping", 500, "1.000", "tri100eigs4k"): 20,
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


def compare_full(got_dir, want_dir, mode, iterations, density):
    """Every CSV the recorded run left, compared as written (empty list: equal)."""
    tag = _tag(mode, iterations, density)
    names = [f"all-{tag}-convergence.csv", f"all-{tag}-construction_status.csv",
             f"all-{tag}-max_backward_iter_150-solver_status.csv",
             f"all-{tag}-max_backward_iter_150-backward_error.csv"]
    problems = []
    for name in names:
        want_path = want_dir / name
        if not want_path.exists():
            continue
        got_path = got_dir / name
        if not got_path.exists():
            problems.append(f"{name}: not written")
            continue
        got, want = _read(got_path), _read(want_path)
        if got == want:
            continue
        for r, (g, w) in enumerate(zip(got, want)):
            if g != w:
                problems.append(f"{name}: row {r}: got {g} want {w}")
                break
        else:
            problems.append(f"{name}: {len(got)} rows, recorded {len(want)}")
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
