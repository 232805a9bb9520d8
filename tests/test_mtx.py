"""The native Matrix Market reader and writer against scipy.io: the reader
must return, bit for bit, the canonical CSC the reference's loader builds
(scripts/common.py:397-402), for every header variant; the writer must read
back to the same bits."""
import os
from pathlib import Path

import numpy as np
import pytest
from scipy import io as spio
from scipy import sparse

from parallellocallyoptimalapproximatesparsematrixinverses_b200 import mtx, problems


def reference_loader(path):
    """scripts/common.py:397-402."""
    a = spio.mmread(path, spmatrix=True).tocsc().astype(np.float64)
    a.sum_duplicates()
    a.eliminate_zeros()
    a.sort_indices()
    return a


def assert_same_csc(got, want):
    assert got.shape == want.shape
    assert np.array_equal(got.indptr, want.indptr)
    assert np.array_equal(got.indices, want.indices)
    assert np.array_equal(got.data.view(np.int64), np.asarray(want.data, np.float64).view(np.int64))


def _random(n, m, density, seed, symmetric=False):
    rng = np.random.default_rng(seed)
    a = sparse.random(n, m, density=density, random_state=rng, format="csc")
    a.data = rng.standard_normal(a.nnz) * 10.0 ** rng.integers(-8, 8, a.nnz)
    if symmetric:
        a = sparse.csc_matrix(sparse.tril(a) + sparse.tril(a, k=-1).T)
    return a


@pytest.mark.parametrize("symmetry", ["general", "symmetric"])
@pytest.mark.parametrize("field", ["real", "integer", "pattern"])
def test_reader_matches_the_reference_loader(tmp_path, symmetry, field):
    a = _random(300, 300, 0.02, 1, symmetric=symmetry == "symmetric")
    if field == "integer":
        a.data = np.round(a.data * 1e3 % 1000)
    path = tmp_path / "a.mtx"
    spio.mmwrite(path, a, field=field, symmetry=symmetry, comment="written by scipy\nsecond comment line")
    assert_same_csc(mtx.load_matrix(path), reference_loader(path))


def test_reader_sums_duplicates_drops_zeros_and_mirrors(tmp_path):
    text = """%%MatrixMarket matrix coordinate real symmetric
% a comment
4 4 7

1 1 2.5
3 1 -1e-3
3 1 4.0
2 2 0.0
4 3 1.25e300
4 4 -7
3 2 0
"""
    path = tmp_path / "d.mtx"
    path.write_text(text.replace("\n", "\r\n"))
    got = mtx.load_matrix(path)
    assert_same_csc(got, reference_loader(path))
    dense = got.toarray()
    assert dense[2, 0] == dense[0, 2] == -1e-3 + 4.0
    assert got.nnz == 6  # (1,1), (3,1), (1,3), (4,3), (3,4), (4,4): both stored zeros leave


def test_reader_skew_symmetric_and_array(tmp_path):
    s = _random(40, 40, 0.1, 3)
    skew = sparse.csc_matrix(sparse.tril(s, k=-1) - sparse.tril(s, k=-1).T)
    path = tmp_path / "skew.mtx"
    spio.mmwrite(path, skew, symmetry="skew-symmetric")
    assert_same_csc(mtx.load_matrix(path), reference_loader(path))
    dense = _random(7, 5, 0.5, 4).toarray()
    path = tmp_path / "array.mtx"
    spio.mmwrite(path, dense)
    want = sparse.csc_matrix(dense)
    want.eliminate_zeros()
    assert_same_csc(mtx.load_matrix(path), want)
    sym = _random(6, 6, 0.6, 5, symmetric=True).toarray()
    path = tmp_path / "array_sym.mtx"
    spio.mmwrite(path, sym, symmetry="symmetric")
    want = sparse.csc_matrix(sym)
    want.eliminate_zeros()
    assert_same_csc(mtx.load_matrix(path), want)


@pytest.mark.parametrize("threads", [1, 3, 16])
def test_parallel_parse_of_a_large_file(tmp_path, threads):
    a = problems.random_banded_spd(60_000, half_width=3, extra=4, seed=2)
    path = tmp_path / "big.mtx"
    spio.mmwrite(path, a, symmetry="symmetric")
    assert os.path.getsize(path) > 4 << 20  # several 1 MiB slices
    assert_same_csc(mtx.load_matrix(path, threads=threads), reference_loader(path))


def test_writer_round_trips_bits(tmp_path):
    a = _random(500, 400, 0.01, 7)
    a.data[::7] = np.nextafter(a.data[::7], np.inf)
    path = mtx.write_matrix(tmp_path / "w.mtx", a)
    assert_same_csc(mtx.load_matrix(path), reference_loader(path))
    assert_same_csc(reference_loader(path), sparse.csc_matrix(a))
    sym = problems.diffusion_2d(12, 1.0, 3)
    path = mtx.write_matrix(tmp_path / "s.mtx", sym, symmetric=True)
    assert path.read_text().startswith("%%MatrixMarket matrix coordinate real symmetric")
    assert_same_csc(mtx.load_matrix(path), sparse.csc_matrix(sym))


def test_preconditioner_save_and_load_layout(tmp_path):
    m = _random(50, 50, 0.1, 9)
    path = mtx.save_preconditioner(tmp_path / "data", "global_spai_mr", m)
    assert path == tmp_path / "data" / "global_spai_mr" / "preconditioner.mtx"
    back = mtx.load_preconditioner(path)
    assert isinstance(back, sparse.csr_matrix)
    want = sparse.csr_matrix(m)
    want.sort_indices()
    assert np.array_equal(back.indptr, want.indptr) and np.array_equal(back.indices, want.indices)
    assert np.array_equal(back.data.view(np.int64), want.data.view(np.int64))


@pytest.mark.parametrize("text,message", [
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", "complex"),
    ("%%MatrixMarket tensor coordinate real general\n", "not a Matrix Market matrix"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n", "expected 2 entries, found 1"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", "out of range"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 x\n", "malformed value"),
    ("%%MatrixMarket matrix coordinate real symmetric\n2 3 0\n", "must be square"),
])
def test_reader_rejects_bad_files(tmp_path, text, message):
    path = tmp_path / "bad.mtx"
    path.write_text(text)
    with pytest.raises(RuntimeError, match=message):
        mtx.load_matrix(path)
    with pytest.raises(RuntimeError, match="cannot open"):
        mtx.load_matrix(tmp_path / "missing.mtx")


SAMPLES = Path(os.environ.get("REFERENCE", "/root/reference")) / "scripts" / "sample_datasets"


@pytest.mark.skipif(not SAMPLES.is_dir(), reason="the reference's sample matrices are not present")
def test_reference_sample_matrices(tmp_path):
    files = sorted(SAMPLES.glob("*.mtx"))
    assert files
    for path in files:
        assert_same_csc(mtx.load_matrix(path), reference_loader(path))
