"""Host supernode partition (swc_supernodes) against the reference's symbolic phase."""
import numpy as np
import pytest

from conftest import SMALL_CASES, load_small


def lib_or_skip():
    import swcholesky_b200 as S
    try:
        S.lib()
    except RuntimeError as e:
        pytest.skip(str(e))
    return S


@pytest.mark.parametrize("name", SMALL_CASES)
def test_column_counts_match_reference(name):
    """With relaxation off, every supernode is exact: the row count of column k inside its
    supernode equals the reference's column count of L (cholesky/sw_LSparsity.h)."""
    S = lib_or_skip()
    d = load_small(name)
    n = int(d["n"])
    bs = S.supernodes(n, d["A2p"], d["A2i"], nrelax=[0, 0, 0], zrelax=[0.0, 0.0, 0.0])
    lay = S.layout(n, d["A2p"], d["A2i"], bs)
    Lip = lay["Li_ptr"].astype(np.int64)
    ours = np.zeros(n, np.int64)
    for s in range(bs.size - 1):
        f, l = bs[s], bs[s + 1]
        nrow = Lip[l] - Lip[f] if l < n else Lip[n] - Lip[f]
        ours[f:l] = nrow - np.arange(l - f)
    np.testing.assert_array_equal(ours, d["colcount"].astype(np.int64))


@pytest.mark.parametrize("name", SMALL_CASES)
def test_relaxed_partition_is_valid(name):
    S = lib_or_skip()
    d = load_small(name)
    n = int(d["n"])
    bs = S.supernodes(n, d["A2p"], d["A2i"])
    assert bs[0] == 0 and bs[-1] == n and np.all(np.diff(bs) > 0)
    lay = S.layout(n, d["A2p"], d["A2i"], bs)
    # relaxed supernodes hold every nonzero of L; the stored size stays within 10% of the
    # reference's relaxed partition (its L has xsize = len(L) doubles)
    nnzL = int(d["colcount"].sum())
    entries = 0
    Lip = lay["Li_ptr"].astype(np.int64)
    for s in range(bs.size - 1):
        f, l = bs[s], bs[s + 1]
        w = l - f
        m = (Lip[l] if l < n else Lip[n]) - Lip[f]
        entries += w * m - w * (w - 1) // 2
    assert nnzL <= entries
    assert lay["xsize"] <= 1.1 * d["L"].size
    wide = S.supernodes(n, d["A2p"], d["A2i"], max_width=16)
    assert np.diff(wide).max() <= 16


def test_bad_input_rejected():
    S = lib_or_skip()
    with pytest.raises(S.SWCError):
        S.supernodes(3, np.array([0, 1, 2, 3]), np.array([0, 7, 2]))


def test_forest_partition_is_per_matrix_partition():
    """The batched path analyses a block-diagonal matrix: its partition is the matrices'
    own partitions side by side (no supernode crosses a matrix)."""
    S = lib_or_skip()
    from swcholesky_b200 import workloads as W
    mats, _ = W.batch_matrices(count=6, seed=2, lo=5, hi=25)
    parts, off, nzo = [], 0, 0
    cs, rs = [], []
    for m in mats:
        parts.append(S.supernodes(m.n, m.indptr, m.indices)[:-1] + off)
        cs.append(np.asarray(m.indptr[:-1]) + nzo)
        rs.append(np.asarray(m.indices) + off)
        off += m.n
        nzo += int(m.indptr[-1])
    cs.append([nzo])
    forest = S.supernodes(off, np.concatenate(cs), np.concatenate(rs))
    np.testing.assert_array_equal(forest, np.concatenate(parts + [[off]]))
