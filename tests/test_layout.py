"""The library's host layout builder reproduces the reference's symbolic layout bit for bit
(Ls, lC, Li_ptr, supernodal etree) and its prune sets as sets."""
import hashlib

import numpy as np
import pytest

from conftest import SMALL_CASES, load_small, load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import matrices as M
from swcholesky_b200 import workloads as W


@pytest.mark.parametrize("name", SMALL_CASES)
def test_layout_matches_reference(name):
    g = load_small(name)
    n = int(g["n"])
    lay = swc.layout(n, g["A2p"], g["A2i"], g["super"])
    assert np.array_equal(lay["Ls"], g["Ls"])
    assert np.array_equal(lay["lC"].astype(np.int64), g["lC"])
    assert np.array_equal(lay["Li_ptr"].astype(np.int64), g["Li_ptr"])
    assert np.array_equal(lay["sparent"], g["sparent"])
    assert np.array_equal(lay["prunePtr"], g["prunePtr"])
    for s in range(g["super"].size - 1):
        a = np.sort(g["pruneSet"][g["prunePtr"][s]:g["prunePtr"][s + 1]])
        b = lay["pruneSet"][lay["prunePtr"][s]:lay["prunePtr"][s + 1]]
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", SMALL_CASES)
def test_permuted_matrix_matches_reference(name):
    g = load_small(name)
    A, _, _ = W.build(name)
    A2 = M.permute_lower(A, g["perm"])
    assert np.array_equal(A2.indptr, g["A2p"])
    assert np.array_equal(A2.indices, g["A2i"])
    assert np.array_equal(A2.data, g["A2x"])


@pytest.mark.parametrize("name", ["grid2d_100", "grid3d_60", "gmrf_500"])
def test_large_layout_digest(name):
    g = load_sym(name)
    A, _, _ = W.build(name)
    prob = W.assemble(A, g["perm"], g["super"])
    assert prob.xsize == int(g["xsize"])
    assert prob.Ls.size == int(g["ls_len"])
    assert hashlib.sha256(prob.Ls.tobytes()).hexdigest() == str(g["ls_sha256"])
    assert prob.pruneSet.size == int(g["prune_len"])
    assert prob.A2p[-1] == int(g["nnz_a2"])


def test_level_schedule_is_topological():
    g = load_small("grid2d_100")
    lay = swc.layout(int(g["n"]), g["A2p"], g["A2i"], g["super"])
    pos = np.empty(g["super"].size - 1, np.int64)
    pos[lay["partition"]] = np.arange(lay["partition"].size)
    lev = np.empty_like(pos)
    for l in range(lay["levelPtr"].size - 1):
        for p in range(lay["levelPtr"][l], lay["levelPtr"][l + 1]):
            lev[lay["partition"][lay["parPtr"][p]:lay["parPtr"][p + 1]]] = l
    par = lay["sparent"]
    ok = par < 0
    assert np.all(lev[~ok] < lev[par[~ok]])


def test_layout_rejects_bad_partition():
    g = load_small("grid2d_20")
    bad = g["super"].copy()
    bad[-1] += 1
    with pytest.raises(swc.SWCError):
        swc.layout(int(g["n"]), g["A2p"], g["A2i"], bad)
