"""The CPU oracle against the reference's recorded outputs.

The reference's sample runs (scripts/results/results_sample) record every
iteration's ||R||_F with 17 significant digits, computed with 256 column
batches.  The oracle in the reference summation order with 256 batches must
reproduce them bit for bit; this pins the oracle (and through the GPU parity
tests, the CUDA library) to the reference's arithmetic."""
import json
from pathlib import Path

import numpy as np
import pytest
from scipy import sparse

from oracle import pyoracle

GOLDEN = Path(__file__).resolve().parent / "golden"

LABELS = {
    "Global CG": ("global_spai", "cg", 2),
    "Global MR": ("global_spai", "mr", 2),
    "Global LOMR": ("global_spai", "lomr", 2),
    "Inner-outer - 2 inner iter MR": ("inner_outer", "mr", 2),
    "Inner-outer - 2 inner iter LOMR": ("inner_outer", "lomr", 2),
    "Inner-outer - 5 inner iter MR": ("inner_outer", "mr", 5),
    "Inner-outer - 5 inner iter LOMR": ("inner_outer", "lomr", 5),
}


def load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    return sparse.csc_matrix((z["data"], z["indices"], z["indptr"]), shape=tuple(z["shape"]))


def golden_sets():
    data = json.loads((GOLDEN / "convergence.json").read_text())
    for key, entry in sorted(data.items()):
        for label, values in entry["histories"].items():
            yield pytest.param(entry, label, [float(v) for v in values], id=f"{key}:{label}")


@pytest.mark.parametrize("entry,label,expected", list(golden_sets()))
def test_history_bit_exact(entry, label, expected):
    family, method, inner = LABELS[label]
    A = load(entry["dataset"])
    n = A.shape[0]
    rows = len(expected)
    if not entry["enable_dropping"] and family == "inner_outer":
        rows = min(rows, 12)  # M fills in quickly without dropping; 11 iterations keep the test short
    result = pyoracle.run(family, method, A, M0=sparse.identity(n, format="csc"),
                          Pr=sparse.diags(1.0 / A.diagonal(), format="csc"), max_iterations=rows - 1,
                          tolerance=1e-9, max_density=entry["max_density"], enable_dropping=entry["enable_dropping"],
                          num_threads=entry["requested_threads"], inner_iterations=inner,
                          order=pyoracle.ORDER_REFERENCE, omp_threads=4)
    got = result.history["residual_norm"]
    want = np.array(expected[:rows])
    k = min(len(got), len(want))
    assert k == len(want), f"history shorter than the recording: {len(got)} < {len(want)}"
    assert np.array_equal(got[:k].view(np.int64), want[:k].view(np.int64)), (
        f"first difference at iteration {int(np.argmax(got[:k] != want[:k]))}")
