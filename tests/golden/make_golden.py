"""Generates the committed golden fixtures from the reference tree.

Run from the repository root with the reference checked out (read-only) at
REFERENCE (default /root/reference) and after `make -C oracle ref`:

    python tests/golden/make_golden.py

Outputs (small, committed):
  <dataset>.npz           A of the sample matrix (canonical CSC, as the
                          reference's scripts/common.py:397-402 loads it)
  convergence.json        the first rows of the reference's recorded
                          per-iteration ||R||_F histories for every method
                          (scripts/results/results_sample/**/*-convergence.csv)
  pcg_reference.npz       histories and statuses of the reference's own PCG
                          (methods_cython/backward_error.pyx compiled into
                          oracle/_ref) on seeded problems, threads = 1
"""
from __future__ import annotations

import csv
import json
import os
import sys
from pathlib import Path

import numpy as np
from scipy import sparse
from scipy.io import mmread

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
REFERENCE = Path(os.environ.get("REFERENCE", "/root/reference"))

SETS = [
    # dataset, dropping dir, max_iter dir, density dir, rows kept
    ("tri100eigs4k", "dropping", 500, "0.030", 41),
    ("tri100eigs4k", "no_dropping", 500, "1.000", 21),
    ("bcsstk21", "dropping", 1000, "0.030", 11),
]


def load_matrix(name: str) -> sparse.csc_matrix:
    a = mmread(REFERENCE / "scripts" / "sample_datasets" / f"{name}-dataset.mtx")
    a = sparse.csc_matrix(a).astype(np.float64)
    a.sum_duplicates()
    a.eliminate_zeros()
    a.sort_indices()
    return a


def main() -> None:
    golden = {}
    for name in sorted({s[0] for s in SETS}):
        a = load_matrix(name)
        np.savez_compressed(HERE / f"{name}.npz", indptr=a.indptr.astype(np.int64),
                            indices=a.indices.astype(np.int64), data=a.data, shape=np.array(a.shape))
    for name, drop, iters, dens, keep in SETS:
        path = (REFERENCE / "scripts" / "results" / "results_sample" / drop / f"max_iter_{iters}" /
                f"max_density_{dens}" / name / f"all-{drop}-max_iter_{iters}-max_density_{dens}-convergence.csv")
        rows = list(csv.reader(path.open()))
        header = rows[0]
        columns = {}
        for ci, label in enumerate(header[1:], start=1):
            values = [float(r[ci]) for r in rows[1:1 + keep] if r[ci] != ""]
            columns[label] = [repr(v) for v in values]
        key = f"{name}/{drop}/max_iter_{iters}/max_density_{dens}"
        golden[key] = {"dataset": name, "enable_dropping": drop == "dropping", "max_density": float(dens),
                       "requested_threads": 256, "source": str(path.relative_to(REFERENCE)), "histories": columns}
    (HERE / "convergence.json").write_text(json.dumps(golden, indent=1))

    # reference PCG (threads = 1) on seeded problems
    from oracle import pyoracle
    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import problems
    ref = pyoracle.reference_pcg_module()
    if ref is None:
        raise SystemExit("build the reference PCG first: make -C oracle ref")
    out = {}
    cases = {
        "diff2d_24_jacobi": (problems.diffusion_2d(24, 1.0, 5), None),
        "lap2d_32_jacobi": (problems.laplacian_2d(32), None),
        "tri4k_jacobi": (load_matrix("tri100eigs4k"), None),
    }
    for label, (a, _) in cases.items():
        a = sparse.csr_matrix(a)
        a.sort_indices()
        m = sparse.csr_matrix(problems.diagonal_inverse(a))
        b, _ = problems.solution_rhs(a, seed=0)
        for tol in (1e-6, 1e-8):
            hist, status = ref.pcg(a.data, a.indices.astype(np.int64), a.indptr.astype(np.int64), m.data,
                                   m.indices.astype(np.int64), m.indptr.astype(np.int64), b, 3000, 1, tol)
            out[f"{label}_tol{tol:g}_history"] = hist
            out[f"{label}_tol{tol:g}_status"] = np.array(status)
    np.savez_compressed(HERE / "pcg_reference.npz", **out)
    print("wrote", sorted(p.name for p in HERE.iterdir()))


if __name__ == "__main__":
    main()
