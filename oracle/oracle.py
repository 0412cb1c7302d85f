"""TEST ORACLE ONLY -- Python access to the two CPU checkers for the CUDA library.

* ``ref_read_matrix``: the reference's Matrix Market reader (readMatrix, common/Util.h).
* ``RefSymbolic`` / ``ref_factor``: the reference's own host symbolic phase (analyze_p2,
  ``cholesky/sw_LSparsity.h:248-702``) and FP64 numeric executor
  (``cholesky/sw_parallel_PB_Cholesky_05_check.c:43-692``), compiled from the reference
  sources into ``oracle/_ref/libswref.so`` by ``oracle/Makefile``.
* ``oracle_factor`` / ``oracle_solve`` / ``oracle_symv``: this project's plain-C restatement
  of the same numeric factor and of the supernodal solves (``oracle/swc_oracle.c``),
  built into ``oracle/build/liboracle_swc.so``.

Only tests, the smoke check and the benchmark's CPU-baseline leg import this module; the
product never does.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libswref.so")
ORACLE_LIB = os.path.join(HERE, "build", "liboracle_swc.so")

_ref = None
_orc = None


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _load_ref():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_LIB)
        lib.swc_ref_analyze.restype = ctypes.c_void_p
        lib.swc_ref_analyze.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + [ctypes.c_int] * 3
        lib.swc_ref_sizes.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.swc_ref_arrays.argtypes = [ctypes.c_void_p] * 16
        lib.swc_ref_factor.restype = ctypes.c_double
        lib.swc_ref_factor.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_int, ctypes.c_void_p]
        lib.swc_ref_free.argtypes = [ctypes.c_void_p]
        lib.swc_ref_read_matrix.restype = ctypes.c_int
        lib.swc_ref_read_matrix.argtypes = [ctypes.c_char_p] + [ctypes.c_void_p] * 5
        lib.swc_ref_free_matrix.argtypes = [ctypes.c_void_p] * 3
        _ref = lib
    return _ref


def _load_oracle():
    global _orc
    if _orc is None:
        lib = ctypes.CDLL(ORACLE_LIB)
        lib.swc_oracle_factor.restype = ctypes.c_int
        lib.swc_oracle_factor.argtypes = ([ctypes.c_int] + [ctypes.c_void_p] * 8 +
                                          [ctypes.c_int] + [ctypes.c_void_p] * 2 +
                                          [ctypes.c_int] + [ctypes.c_void_p] * 4)
        lib.swc_oracle_solve.argtypes = ([ctypes.c_int] + [ctypes.c_void_p] * 5 +
                                         [ctypes.c_int, ctypes.c_void_p, ctypes.c_int])
        lib.swc_oracle_symv.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 5
        _orc = lib
    return _orc


@dataclass
class Symbolic:
    """Every array of the supernodal structure, in the reference's conventions."""
    n: int
    nsuper: int
    xsize: int
    perm: np.ndarray        # final permutation (after the weighted postorder)
    colcount: np.ndarray    # exact column counts of L (permuted order)
    super: np.ndarray       # blockSet, nsuper+1
    sparent: np.ndarray     # supernodal etree (-1 = root)
    Ls: np.ndarray          # row lists
    lC: np.ndarray          # column value offsets (int64, n+1)
    Li_ptr: np.ndarray      # column row-list offsets (int64, n+1)
    A2p: np.ndarray
    A2i: np.ndarray
    A2x: np.ndarray
    prunePtr: np.ndarray
    pruneSet: np.ndarray
    levelPtr: np.ndarray
    parPtr: np.ndarray
    partition: np.ndarray
    maxSupWid: int
    maxCol: int
    symbolic_seconds: float

    @property
    def nLevels(self) -> int:
        return int(self.levelPtr.size - 1)

    @property
    def flops(self) -> float:
        """fl = sum_j c_j^2 over exact column counts (cholesky/ColumnCount.h:492-498)."""
        c = self.colcount.astype(np.float64)
        return float(np.sum(c * c))


class RefSymbolic:
    """Handle on the reference's analysed structure (owns the C-side state)."""

    def __init__(self, A, perm, cost_param: int = 64, level_param: int = -1,
                 final_seq_node: int = 4):
        lib = _load_ref()
        perm = np.ascontiguousarray(perm, dtype=np.int64)
        self._lib = lib
        self._h = lib.swc_ref_analyze(int(A.n), _p(A.indptr), _p(A.indices), _p(A.data),
                                      _p(perm), cost_param, level_param, final_seq_node)
        if not self._h:
            raise RuntimeError("reference analyze_p2 failed")
        sz = np.zeros(12, dtype=np.int64)
        lib.swc_ref_sizes(self._h, _p(sz))
        n, ns, xs, nls, nnz2, nlev, nparts, npart, nprune, msw, mcol, us = (int(v) for v in sz)
        a = dict(
            perm=np.zeros(n, np.int32), colcount=np.zeros(n, np.int32),
            super=np.zeros(ns + 1, np.int32), sparent=np.zeros(ns, np.int32),
            Ls=np.zeros(nls, np.int32), lC=np.zeros(n + 1, np.int64),
            Li_ptr=np.zeros(n + 1, np.int64), A2p=np.zeros(n + 1, np.int32),
            A2i=np.zeros(nnz2, np.int32), A2x=np.zeros(nnz2, np.float64),
            prunePtr=np.zeros(ns + 1, np.int32), pruneSet=np.zeros(nprune, np.int32),
            levelPtr=np.zeros(nlev + 1, np.int32), parPtr=np.zeros(nparts + 1, np.int32),
            partition=np.zeros(npart, np.int32))
        lib.swc_ref_arrays(self._h, *[_p(a[k]) for k in (
            "perm", "colcount", "super", "sparent", "Ls", "lC", "Li_ptr", "A2p", "A2i",
            "A2x", "prunePtr", "pruneSet", "levelPtr", "parPtr", "partition")])
        self.sym = Symbolic(n=n, nsuper=ns, xsize=xs, maxSupWid=msw, maxCol=mcol,
                            symbolic_seconds=us * 1e-6, **a)

    def factor(self, values=None, threads: int = 0):
        """Runs the reference FP64 executor; returns (lValues, seconds, return value)."""
        L = np.zeros(self.sym.xsize, dtype=np.float64)
        ret = ctypes.c_int(0)
        vals = None if values is None else np.ascontiguousarray(values, dtype=np.float64)
        t = self._lib.swc_ref_factor(self._h, _p(vals), _p(L), int(threads), ctypes.byref(ret))
        return L, float(t), int(ret.value)

    def close(self):
        if self._h:
            self._lib.swc_ref_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_read_matrix(path):
    """The reference's readMatrix (common/Util.h:77-179) on a file: (n, indptr, indices,
    data) of the lower CSC matrix it builds, or None when it reports failure."""
    lib = _load_ref()
    n, nnz = ctypes.c_longlong(0), ctypes.c_longlong(0)
    c, r = ctypes.POINTER(ctypes.c_int)(), ctypes.POINTER(ctypes.c_int)()
    v = ctypes.POINTER(ctypes.c_double)()
    if not lib.swc_ref_read_matrix(os.fsencode(path), ctypes.byref(n), ctypes.byref(nnz),
                                   ctypes.byref(c), ctypes.byref(r), ctypes.byref(v)):
        return None
    nn, nz = int(n.value), int(nnz.value)
    out = (nn, np.ctypeslib.as_array(c, shape=(nn + 1,)).copy(),
           np.ctypeslib.as_array(r, shape=(nz,)).copy(),
           np.ctypeslib.as_array(v, shape=(nz,)).copy())
    lib.swc_ref_free_matrix(ctypes.cast(c, ctypes.c_void_p), ctypes.cast(r, ctypes.c_void_p),
                            ctypes.cast(v, ctypes.c_void_p))
    return out


def oracle_factor(n, A2p, A2i, A2x, lC, Ls, Li_ptr, super_, prunePtr, pruneSet, levelPtr,
                  parPtr, partition, xsize):
    """Runs the C restatement; returns (lValues, ok, info)."""
    lib = _load_oracle()
    L = np.zeros(int(xsize), dtype=np.float64)
    info = ctypes.c_int(0)
    arrs = [np.ascontiguousarray(x) for x in (A2p, A2i, A2x, lC, Ls, Li_ptr, super_,
                                              prunePtr, pruneSet, levelPtr, parPtr, partition)]
    A2p, A2i, A2x, lC, Ls, Li_ptr, super_, prunePtr, pruneSet, levelPtr, parPtr, partition = arrs
    ok = lib.swc_oracle_factor(int(n), _p(A2p), _p(A2i), _p(A2x), _p(lC), _p(Ls), _p(Li_ptr),
                               _p(L), _p(super_), int(super_.size - 1), _p(prunePtr),
                               _p(pruneSet), int(levelPtr.size - 1), _p(levelPtr), _p(parPtr),
                               _p(partition), ctypes.byref(info))
    return L, int(ok), int(info.value)


def oracle_solve(n, lC, Ls, Li_ptr, L, super_, b):
    """x = (L L^T)^{-1} b in the permuted ordering; b is (n,) or (n, nrhs)."""
    lib = _load_oracle()
    b = np.asarray(b, dtype=np.float64)
    x = np.array(b.reshape(n, -1), order="F", copy=True)
    lC = np.ascontiguousarray(lC, np.int64)
    Ls = np.ascontiguousarray(Ls, np.int32)
    Li_ptr = np.ascontiguousarray(Li_ptr, np.int64)
    super_ = np.ascontiguousarray(super_, np.int32)
    L = np.ascontiguousarray(L, np.float64)
    lib.swc_oracle_solve(int(n), _p(lC), _p(Ls), _p(Li_ptr), _p(L), _p(super_),
                         int(super_.size - 1), _p(x), int(x.shape[1]))
    return x.reshape(b.shape)


def oracle_symv(n, A2p, A2i, A2x, x):
    lib = _load_oracle()
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(n, np.float64)
    A2p = np.ascontiguousarray(A2p, np.int32)
    A2i = np.ascontiguousarray(A2i, np.int32)
    A2x = np.ascontiguousarray(A2x, np.float64)
    lib.swc_oracle_symv(int(n), _p(A2p), _p(A2i), _p(A2x), _p(x), _p(y))
    return y
