"""Generates the golden fixtures under tests/golden/ from the reference itself.

Runs the reference's own host symbolic phase (analyze_p2) and FP64 numeric executor, built
from the reference sources by oracle/Makefile into oracle/_ref/libswref.so, on the seeded
synthetic workloads, and stores what the tests and the benchmark need where the reference
is not available:

* ``small_<name>.npz`` -- small cases: every symbolic array the reference's numeric phase
  consumes (A2, BCSC layout, prune sets in the reference's order, H-level schedule), the
  reference's factor L, and a seeded right-hand side.  These pin the oracle and the GPU.
* ``sym_<name>.npz`` -- large workloads: the reference's final permutation (after its
  weighted postorder), its supernode partition, and checks on the derived structure (xsize,
  length and SHA-256 of Ls, flop count fl = sum_j c_j^2 and nnz(L) = sum_j c_j from its
  exact column counts).  The
  matrix values are regenerated from the seeded generators; the layout is rebuilt from the
  partition with the library's layout builder and checked against these values.

Usage: python tests/golden/make_golden.py [names...]   (needs the reference checkout)
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from swcholesky_b200 import workloads as W  # noqa: E402

SMALL = ["grid2d_20", "grid3d_8", "stencil27_4", "grid2d_100"]
LARGE = ["grid2d_100", "grid3d_60", "stencil27_40", "gmrf_500", "grid3d_24", "stencil27_12"]


def ls_digest(Ls: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(Ls, np.int32).tobytes()).hexdigest()


def make(name: str):
    A, perm, _ = W.build(name)
    R = O.RefSymbolic(A, perm)
    s = R.sym
    if name in SMALL:
        L, t, ret = R.factor(threads=1)
        assert ret == 1
        b = np.random.default_rng(0).standard_normal(s.n)
        np.savez_compressed(
            os.path.join(HERE, f"small_{name}.npz"), n=s.n, perm=s.perm, colcount=s.colcount,
            super=s.super, sparent=s.sparent, Ls=s.Ls, lC=s.lC, Li_ptr=s.Li_ptr, A2p=s.A2p,
            A2i=s.A2i, A2x=s.A2x, prunePtr=s.prunePtr, pruneSet=s.pruneSet,
            levelPtr=s.levelPtr, parPtr=s.parPtr, partition=s.partition, L=L, b=b,
            maxSupWid=s.maxSupWid, maxCol=s.maxCol, fl=s.flops)
        print(f"small_{name}: n={s.n} nsuper={s.nsuper} xsize={s.xsize}")
    if name in LARGE:
        np.savez_compressed(
            os.path.join(HERE, f"sym_{name}.npz"), n=s.n, perm=s.perm, super=s.super,
            xsize=s.xsize, ls_len=s.Ls.size, ls_sha256=ls_digest(s.Ls), fl=s.flops,
            nnzl=int(s.colcount.astype(np.int64).sum()), nnz_a2=s.A2p[-1],
            prune_len=s.pruneSet.size, maxSupWid=s.maxSupWid)
        print(f"sym_{name}: n={s.n} nsuper={s.nsuper} xsize={s.xsize} fl={s.flops:.4g}")
    R.close()


if __name__ == "__main__":
    names = sys.argv[1:] or sorted(set(SMALL) | set(LARGE))
    for nm in names:
        make(nm)
