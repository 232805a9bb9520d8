"""The reference's own, unmodified Cython binding (methods_cython/methods.pyx),
compiled against include/methods_c_api.h and linked to libspai_b200.so by
oracle/build_relink.sh, replays the reference's recorded runs bit for bit:
the relink a user of the reference makes to switch to this library."""
import importlib.util
import json
from pathlib import Path

import numpy as np
import pytest
from scipy import sparse

from parallellocallyoptimalapproximatesparsematrixinverses_b200 import global_spai, inner_outer, problems
from tests.helpers import assert_same_result

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
RELINKED = ROOT / "oracle" / "_ref" / "relinked"
LABELS = {
    "Global CG": ("global_spai", "cg", 2),
    "Global MR": ("global_spai", "mr", 2),
    "Global LOMR": ("global_spai", "lomr", 2),
    "Inner-outer - 2 inner iter MR": ("inner_outer", "mr", 2),
    "Inner-outer - 5 inner iter LOMR": ("inner_outer", "lomr", 5),
}


def _relinked():
    paths = sorted(RELINKED.glob("methods*.so"))
    if not paths:
        pytest.fail("oracle/_ref/relinked is not built: run `make -C oracle relink` where the reference tree is "
                    "present (build() does) before the GPU tests")
    spec = importlib.util.spec_from_file_location("methods", paths[0])
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def _load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    return sparse.csc_matrix((z["data"], z["indices"], z["indptr"]), shape=tuple(z["shape"]))


def _recorded():
    data = json.loads((GOLDEN / "convergence.json").read_text())
    for key, entry in sorted(data.items()):
        if not entry["enable_dropping"]:
            continue
        for label, values in entry["histories"].items():
            if label in LABELS:
                yield pytest.param(entry, label, [float(v) for v in values], id=f"{key}:{label}")


@pytest.mark.gpu
@pytest.mark.parametrize("entry,label,expected", list(_recorded()))
def test_relinked_binding_replays_the_recorded_histories(require_gpu, entry, label, expected):
    methods = _relinked()
    family, name, inner = LABELS[label]
    A = _load(entry["dataset"])
    n = A.shape[0]
    rows = min(len(expected), 60)
    kw = dict(M0=sparse.identity(n, format="csc"), Pr=sparse.diags(1.0 / A.diagonal(), format="csc"),
              max_iterations=rows - 1, tolerance=1e-9, max_density=entry["max_density"],
              enable_dropping=entry["enable_dropping"], num_threads=entry["requested_threads"])
    if family == "inner_outer":
        kw["inner_iterations"] = inner
    got = getattr(getattr(methods, family), name)(A, **kw).history["residual_norm"]
    want = np.array(expected[:rows])
    assert np.array_equal(got[:rows].view(np.int64), want.view(np.int64)), (
        f"first difference at iteration {int(np.argmax(got[:rows] != want))}")


@pytest.mark.gpu
def test_relinked_binding_matches_the_package_surface(require_gpu):
    methods = _relinked()
    A = problems.diffusion_2d(20, 1.0, 8)
    M0 = problems.diagonal_inverse(A)
    for family, ours in (("global_spai", global_spai), ("inner_outer", inner_outer)):
        for name in getattr(methods, family).available_methods:
            kw = dict(M0=M0, max_iterations=6, tolerance=1e-12, max_density=0.03, num_threads=3)
            got = getattr(getattr(methods, family), name)(A, **kw)
            want = getattr(ours, name)(A, **kw)
            assert_same_result(got, want, f"{family}.{name}")
    with pytest.raises(RuntimeError, match="Invalid threads count value"):
        methods.global_spai.mr(A, num_threads=0)
