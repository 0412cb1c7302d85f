"""Matrix Market reader/writer, permutation files and the general-graph nested dissection
(host-only entry points of the library; no GPU).

Parity: on well-formed files the library's reader gives exactly the lower CSC matrix the
reference's readMatrix (common/Util.h:77-179, run from oracle/_ref) builds; files the
reference cannot read (unsorted, duplicated or upper-triangle entries, general symmetric
files, empty columns) give the matrix a careful reader must give, checked against scipy.
The ordering must be a permutation, accepted by the reference's analyze_p2, and reduce the
fill (sum of squared column counts) far below the natural order."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import swcholesky_b200 as swc
from swcholesky_b200 import matrices as M
from oracle import oracle as O


def lower_of(mat):
    low = sp.csc_matrix(sp.tril(sp.csc_matrix(mat)))
    low.sum_duplicates()
    low.sort_indices()
    return low


def write_lines(path, lines):
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def test_roundtrip_and_reference_reader(tmp_path):
    A = M.random_geometric(2000, dim=2, degree=8, seed=3)
    f = str(tmp_path / "a.mtx")
    swc.write_mtx(f, A.n, A.indptr, A.indices, A.data)
    B = swc.read_mtx(f)
    assert B.n == A.n
    assert np.array_equal(B.indptr, A.indptr) and np.array_equal(B.indices, A.indices)
    assert np.array_equal(B.data, A.data)     # %.17g round-trips doubles exactly
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    n, c, r, v = O.ref_read_matrix(f)
    assert n == A.n
    assert np.array_equal(c, B.indptr) and np.array_equal(r, B.indices)
    assert np.array_equal(v, B.data)


def test_careful_reading(tmp_path):
    # 4 x 4 SPD matrix given out of order, with a duplicate, an upper entry, comments,
    # blank lines, CRLF endings, an upper-case header and the "integer" field
    f = str(tmp_path / "b.mtx")
    lines = ["%%MATRIXMARKET Matrix Coordinate Integer Symmetric",
             "% comment", "", "4 4 7",
             "3 3 5", "1 1 4", "2 1 -1", "% inside", "1 2 -1", "2 2 3", "4 4 2", "4 3 1"]
    with open(f, "w", newline="") as fh:
        fh.write("\r\n".join(lines) + "\r\n")
    B = swc.read_mtx(f)
    dense = np.zeros((4, 4))
    for j in range(4):
        for p in range(B.indptr[j], B.indptr[j + 1]):
            dense[B.indices[p], j] = B.data[p]
    expect = np.array([[4, 0, 0, 0], [-2, 3, 0, 0], [0, 0, 5, 0], [0, 0, 1, 2]], float)
    assert np.array_equal(dense, expect)     # (2,1) given twice (once as (1,2)): summed
    for j in range(4):                        # sorted rows, diagonal first
        rows = B.indices[B.indptr[j]:B.indptr[j + 1]]
        assert rows[0] == j and np.all(np.diff(rows) > 0)


def test_general_file_and_empty_column(tmp_path):
    rng = np.random.default_rng(0)
    X = sp.random(30, 30, density=0.1, random_state=1)
    S = (X + X.T + 30 * sp.identity(30)).tocoo()
    f = str(tmp_path / "g.mtx")
    lines = ["%%MatrixMarket matrix coordinate real general", f"30 30 {S.nnz}"]
    order = rng.permutation(S.nnz)
    lines += [f"{S.row[k] + 1} {S.col[k] + 1} {float(S.data[k])!r}" for k in order]
    write_lines(f, lines)
    B = swc.read_mtx(f)
    ref = lower_of(S)
    assert np.array_equal(B.indptr, ref.indptr) and np.array_equal(B.indices, ref.indices)
    assert np.allclose(B.data, ref.data, rtol=0, atol=0)
    # a column with no entry at all, and a missing diagonal: explicit zero diagonals
    f2 = str(tmp_path / "e.mtx")
    write_lines(f2, ["%%MatrixMarket matrix coordinate real symmetric", "3 3 2", "1 1 2",
                     "3 1 1"])
    E = swc.read_mtx(f2)
    assert list(E.indptr) == [0, 2, 3, 4]
    assert list(E.indices) == [0, 2, 1, 2]
    assert list(E.data) == [2.0, 1.0, 0.0, 0.0]


@pytest.mark.parametrize("lines,msg", [
    (["%%MatrixMarket matrix coordinate complex symmetric", "2 2 1", "1 1 1 0"], "field"),
    (["%%MatrixMarket matrix coordinate pattern symmetric", "2 2 1", "1 1"], "field"),
    (["%%MatrixMarket matrix coordinate real hermitian", "2 2 1", "1 1 1"], "symmetry"),
    (["%%MatrixMarket matrix array real symmetric", "2 2", "1", "2", "3"], "coordinate"),
    (["%%MatrixMarket matrix coordinate real symmetric", "2 3 1", "1 1 1"], "square"),
    (["%%MatrixMarket matrix coordinate real symmetric", "2 2 1", "3 1 1"], "out of range"),
    (["%%MatrixMarket matrix coordinate real symmetric", "2 2 3", "1 1 1", "2 2 1"], "ends after"),
    (["%%MatrixMarket matrix coordinate real symmetric", "2 2 1", "1 1 1", "2 2 1"], "more entries"),
    (["%%MatrixMarket matrix coordinate real general", "2 2 3", "1 1 1", "2 1 1", "1 2 2"],
     "not symmetric"),
    (["%%MatrixMarket matrix coordinate real general", "2 2 2", "1 1 1", "2 1 1"],
     "not symmetric"),
    (["MatrixMarket matrix coordinate real symmetric", "2 2 1", "1 1 1"], "first token"),
    (["%%MatrixMarket matrix coordinate real symmetric", "2 2 1", "1 1 x"], "missing value"),
])
def test_malformed_files_rejected(tmp_path, lines, msg):
    f = str(tmp_path / "bad.mtx")
    write_lines(f, lines)
    with pytest.raises(swc.SWCError) as e:
        swc.read_mtx(f)
    assert e.value.code == swc.SWC_INVALID_INPUT
    assert msg in str(e.value)


def test_perm_files(tmp_path):
    rng = np.random.default_rng(1)
    perm = rng.permutation(1000)
    f = str(tmp_path / "p.bin")
    swc.write_perm(f, perm)
    # the reference's layout: n native size_t values, read with fread
    assert os.path.getsize(f) == 1000 * 8
    assert np.array_equal(np.fromfile(f, dtype=np.uintp), perm)
    assert np.array_equal(swc.read_perm(f, 1000), perm)
    with pytest.raises(swc.SWCError, match="holds 1000 of 1001"):
        swc.read_perm(f, 1001)
    with pytest.raises(swc.SWCError, match="longer"):
        swc.read_perm(f, 999)
    bad = perm.copy()
    bad[3] = bad[4]
    bad.astype(np.uintp).tofile(f)
    with pytest.raises(swc.SWCError, match="permutation"):
        swc.read_perm(f, 1000)
    with pytest.raises(swc.SWCError, match="permutation"):
        swc.write_perm(str(tmp_path / "q.bin"), bad)


def fill(A, perm):
    """sum_j c_j^2 over the exact column counts of the factor of P A P^T (the library's
    supernode partition without relaxation, whose supernodes hold exact columns)."""
    B = M.permute_lower(A, np.asarray(perm))
    sup = swc.supernodes(B.n, B.indptr, B.indices, nrelax=[0, 0, 0], zrelax=[0.0, 0.0, 0.0])
    lip = swc.layout(B.n, B.indptr, B.indices, sup)["Li_ptr"].astype(np.int64)
    tot = 0.0
    for s in range(sup.size - 1):
        f, l = int(sup[s]), int(sup[s + 1])
        k = np.arange(l - f, dtype=np.float64)
        tot += float(np.sum((lip[l] - lip[f] - k) ** 2))
    return tot


@pytest.mark.parametrize("kind", ["rgg2", "rgg3", "grid3"])
def test_nested_dissection_fill(kind):
    if kind == "rgg2":
        A = M.random_geometric(8000, dim=2, degree=8, seed=5)
    elif kind == "rgg3":
        A = M.random_geometric(8000, dim=3, degree=10, seed=6)
    else:
        A = M.laplacian_3d(20, 1e-3)
    perm = swc.order_nd(A.n, A.indptr, A.indices)
    assert np.array_equal(np.sort(perm), np.arange(A.n))
    f_nd, f_nat = fill(A, perm), fill(A, np.arange(A.n))
    # the natural order of a grid is already banded; of a random graph it is not
    assert f_nd < (0.2 if kind == "grid3" else 0.05) * f_nat, (f_nd, f_nat)
    if kind == "grid3":   # no worse than the geometric dissection of the grid
        assert f_nd <= fill(A, M.nested_dissection((20, 20, 20)))


def test_nested_dissection_special_graphs():
    # disconnected pieces, an isolated vertex, a complete subgraph above the leaf size
    blocks = [sp.csc_matrix(M.laplacian_2d(12).to_scipy_full()),
              sp.csc_matrix(np.ones((100, 100)) + 100 * np.eye(100)),
              sp.identity(1, format="csc")]
    A = M.LowerCSC.from_scipy(sp.block_diag(blocks))
    for leaf in (0, 8, 64):
        perm = swc.order_nd(A.n, A.indptr, A.indices, leaf=leaf)
        assert np.array_equal(np.sort(perm), np.arange(A.n))
    one = M.LowerCSC.from_scipy(sp.identity(1, format="csc"))
    assert list(swc.order_nd(1, one.indptr, one.indices)) == [0]


def test_reference_analysis_accepts_the_ordering(tmp_path):
    """The file path of the reference's driver: matrix file -> ordering -> permutation file
    -> the reference's analyze_p2 (GIVEN) -> the library's layout of the same partition is
    the reference's, bit for bit."""
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    A = M.random_geometric(6000, dim=3, degree=10, seed=7)
    fm, fp = str(tmp_path / "r.mtx"), str(tmp_path / "r.perm")
    swc.write_mtx(fm, A.n, A.indptr, A.indices, A.data)
    B = swc.read_mtx(fm)
    swc.write_perm(fp, swc.order_nd(B.n, B.indptr, B.indices))
    perm = swc.read_perm(fp, B.n)
    R = O.RefSymbolic(M.LowerCSC(B.n, B.indptr, B.indices, B.data), perm)
    s = R.sym
    R.close()
    lay = swc.layout(s.n, s.A2p, s.A2i, s.super)
    assert np.array_equal(lay["Ls"], s.Ls)
    assert np.array_equal(lay["lC"].astype(np.int64), s.lC.astype(np.int64))
    assert int(lay["xsize"]) == s.xsize
