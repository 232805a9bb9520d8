"""The device library in the reference's summation order (num_threads column
batches, sums sequential through each batch) replays the reference's own
recorded runs -- the per-iteration ||R||_F of scripts/results/results_sample,
17 significant digits -- bit for bit, and matches the oracle in the reference
order on further cases.  A call with only the reference's arguments goes
through the five methods_c_api.h entry points, which run in this order by
default: the replays below use exactly that drop-in path."""
import json
from pathlib import Path

import numpy as np
import pytest
from scipy import sparse

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import global_spai, inner_outer, problems
from tests.helpers import METHODS, assert_same_result

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
FAMILIES = {"global_spai": global_spai, "inner_outer": inner_outer}
LABELS = {
    "Global CG": ("global_spai", "cg", 2),
    "Global MR": ("global_spai", "mr", 2),
    "Global LOMR": ("global_spai", "lomr", 2),
    "Inner-outer - 2 inner iter MR": ("inner_outer", "mr", 2),
    "Inner-outer - 2 inner iter LOMR": ("inner_outer", "lomr", 2),
    "Inner-outer - 5 inner iter MR": ("inner_outer", "mr", 5),
    "Inner-outer - 5 inner iter LOMR": ("inner_outer", "lomr", 5),
}


def _load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    return sparse.csc_matrix((z["data"], z["indices"], z["indptr"]), shape=tuple(z["shape"]))


def _recorded():
    data = json.loads((GOLDEN / "convergence.json").read_text())
    for key, entry in sorted(data.items()):
        for label, values in entry["histories"].items():
            yield pytest.param(entry, label, [float(v) for v in values], id=f"{key}:{label}")


@pytest.mark.parametrize("entry,label,expected", list(_recorded()))
def test_device_replays_the_recorded_histories(require_gpu, entry, label, expected):
    family, name, inner = LABELS[label]
    A = _load(entry["dataset"])
    n = A.shape[0]
    rows = len(expected)
    if not entry["enable_dropping"] and family == "inner_outer":
        rows = min(rows, 12)
    kw = dict(M0=sparse.identity(n, format="csc"), Pr=sparse.diags(1.0 / A.diagonal(), format="csc"),
              max_iterations=rows - 1, tolerance=1e-9, max_density=entry["max_density"],
              enable_dropping=entry["enable_dropping"], num_threads=entry["requested_threads"])
    if family == "inner_outer":
        kw["inner_iterations"] = inner
    # no extension keyword: the reference's own C entry point (spai_global_cg, ...), default order
    got = getattr(FAMILIES[family], name)(A, **kw).history["residual_norm"]
    want = np.array(expected[:rows])
    assert len(got) >= len(want), f"history shorter than the recording: {len(got)} < {len(want)}"
    assert np.array_equal(got[:rows].view(np.int64), want.view(np.int64)), (
        f"first difference at iteration {int(np.argmax(got[:rows] != want))}")


@pytest.mark.parametrize("family,name", METHODS)
@pytest.mark.parametrize("threads,summation", [(1, "reference"), (7, "reference"), (1, None), (5, None)])
def test_reference_order_matches_the_oracle(require_gpu, family, name, threads, summation):
    A = problems.diffusion_2d(14, 1.0, 6)
    kw = dict(max_iterations=8, tolerance=1e-12, max_density=0.02, num_threads=threads)
    if summation is not None:
        kw["summation"] = summation  # spai_run_ex; without it the reference's own entry point runs
    got = getattr(FAMILIES[family], name)(A, M0=problems.diagonal_inverse(A), **kw)
    kw.pop("summation", None)
    want = pyoracle.run(family, name, A, M0=problems.diagonal_inverse(A), order=pyoracle.ORDER_REFERENCE,
                        omp_threads=2, **kw)
    assert_same_result(got, want, f"{family}.{name} threads={threads}")
