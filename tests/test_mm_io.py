"""Matrix Market input (the source the reference declares with -P/-D/-M but
never reads, solver_collection.cpp:505-601): the library's reader against
scipy.io.mmread on general, symmetric, skew-symmetric, integer and pattern
files, repeated entries and malformed input. CPU only."""
import io

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from solver_cpp_b200 import _abi


def _ref_csr(path):
    M = scipy.io.mmread(str(path), spmatrix=False).tocsr()
    M.sum_duplicates()
    M.sort_indices()
    return M


def _check_equal(A, M):
    assert A.n == M.shape[0]
    assert np.array_equal(A.ptr, M.indptr)
    assert np.array_equal(A.col, M.indices)
    assert np.array_equal(A.val, M.data)


def _random(n, density, seed, symmetric=False):
    rng = np.random.default_rng(seed)
    M = sp.random(n, n, density=density, random_state=rng, format="coo")
    M.data = rng.standard_normal(M.nnz)
    if symmetric:
        M = sp.triu(M) + sp.triu(M, 1).T
    return M


@pytest.mark.parametrize("symmetry", ["general", "symmetric"])
def test_mm_real_matches_scipy(ks, tmp_path, symmetry):
    M = _random(300, 0.02, 1, symmetric=symmetry == "symmetric")
    path = tmp_path / "a.mtx"
    scipy.io.mmwrite(str(path), M, symmetry=symmetry, precision=17)
    assert symmetry in path.read_text().splitlines()[0]
    _check_equal(ks.mm_read(str(path)), _ref_csr(path))


def test_mm_skew_integer_pattern_and_repeats(ks, tmp_path):
    skew = tmp_path / "skew.mtx"
    skew.write_text("%%MatrixMarket matrix coordinate real skew-symmetric\n% a comment\n\n"
                    "4 4 3\n2 1 1.5\n4 1 -2\n3 2 0.25\n")
    _check_equal(ks.mm_read(str(skew)), _ref_csr(skew))
    A = ks.mm_read(str(skew)).to_scipy().toarray()
    assert np.array_equal(A, -A.T)

    integer = tmp_path / "int.mtx"
    integer.write_text("%%MatrixMarket matrix coordinate integer general\n3 3 4\n1 1 5\n2 3 -7\n3 1 2\n3 3 9\n")
    _check_equal(ks.mm_read(str(integer)), _ref_csr(integer))

    pattern = tmp_path / "pat.mtx"
    pattern.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 3\n1 1\n2 1\n3 3\n")
    A = ks.mm_read(str(pattern))
    assert np.array_equal(A.to_scipy().toarray(), np.array([[1, 1, 0], [1, 0, 0], [0, 0, 1.0]]))

    # repeated positions are summed, in file order; rows come out ordered by column
    rep = tmp_path / "rep.mtx"
    rep.write_text("%%MatrixMarket matrix coordinate real general\n2 2 5\n2 2 1e16\n1 2 3\n2 2 1.0\n1 1 4\n"
                   "2 2 -1e16\n")
    A = ks.mm_read(str(rep))
    assert list(A.ptr) == [0, 2, 3] and list(A.col) == [0, 1, 1]
    assert A.val[2] == (1e16 + 1.0) - 1e16 == 0.0  # file order; (1e16 - 1e16) + 1.0 would give 1.0


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1 0\n",
    "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",
    "%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n3 1 1\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n",
    "%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n1 1 1\n",
    "not a matrix market file\n",
])
def test_mm_rejects_malformed(ks, tmp_path, text):
    path = tmp_path / "bad.mtx"
    path.write_text(text)
    with pytest.raises(ks.KrylovError) as e:
        ks.mm_read(str(path))
    assert e.value.status == _abi.KS_BAD_INPUT


def test_mm_missing_file(ks, tmp_path):
    with pytest.raises(ks.KrylovError) as e:
        ks.mm_read(str(tmp_path / "none.mtx"))
    assert e.value.status == _abi.KS_IO_ERROR
