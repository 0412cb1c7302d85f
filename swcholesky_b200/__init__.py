"""swcholesky_b200 -- supernodal sparse Cholesky numeric factorization on NVIDIA B200.

Host-side mirror of the reference's numeric-phase interface over the C ABI of
``libswchol_b200.so`` (``include/swcholesky_b200.h``):

* ``sw_cholesky_left_par_05`` -- the reference entry point
  (``cholesky/sw_parallel_PB_Cholesky_05.h:52-66``) with the same argument names and
  meaning, taking numpy arrays; returns 1 on success and 0 on failure.
* ``Handle`` -- device-resident factorization (analyze once, factor many times, keep L on
  the GPU).
* ``layout`` -- the BCSC layout, prune sets and a level schedule for a supernode partition.

The CUDA library is the only compute path: importing works without a GPU, but every
numeric call raises if the library is missing or no CUDA device is present.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["lib", "SWCError", "sw_cholesky_left_par_05", "Handle", "layout", "LIB_PATH",
           "SWC_OK", "SWC_NOT_SPD", "SWC_MODE_FP64", "read_mtx", "write_mtx", "read_perm",
           "write_perm", "order_nd", "MtxMatrix"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libswchol_b200.so")

SWC_OK = 0
SWC_NOT_SPD = 1
SWC_INVALID_INPUT = 2
SWC_CUDA_ERROR = 3
SWC_STRUCTURE_ERROR = 4
SWC_NOT_READY = 5
SWC_TIMEOUT = 6
DEFAULT_WAIT_BUDGET = 1 << 24
SWC_MODE_FP64 = 0
SWC_MODE_MIXED_TF32X3 = 1
SWC_MODE_MIXED_BF16X3 = 2

# every symbol include/swcholesky_b200.h declares
EXPORTS = (
    "sw_cholesky_left_par_05", "swc_last_info", "swc_last_error", "swc_create", "swc_destroy",
    "swc_set_stream", "swc_get_stream", "swc_analyze", "swc_factor", "swc_get_L",
    "swc_device_L", "swc_sizes", "swc_profile", "swc_plan_stats", "swc_layout_sizes",
    "swc_layout", "swc_solve", "swc_refine", "swc_solve_noalloc", "swc_logdet",
    "swc_logdet_grad", "swc_solve_grad", "swc_supernodes", "swc_batch_analyze",
    "swc_batch_autotune", "swc_batch_berr", "swc_set_plan", "swc_set_wait_budget",
    "swc_read_mtx", "swc_free", "swc_write_mtx", "swc_read_perm", "swc_write_perm",
    "swc_order_nd",
)
KERNEL_CLASSES = ("memset", "small", "assemble", "update", "panel", "syrk")

_lib = None
_VP = ctypes.c_void_p
_I = ctypes.c_int


class SWCError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"swc error {code}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Loads libswchol_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m swcholesky_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        L.sw_cholesky_left_par_05.restype = _I
        L.sw_cholesky_left_par_05.argtypes = ([_I] + [_VP] * 8 + [_I, _VP, _VP, _VP, _I] +
                                              [_VP] * 2 + [_I] + [_VP] * 2 + [_I] * 4 + [_VP])
        L.swc_last_info.restype = _I
        L.swc_last_error.restype = ctypes.c_char_p
        L.swc_create.argtypes = [ctypes.POINTER(_VP), _I]
        L.swc_destroy.argtypes = [_VP]
        L.swc_set_stream.argtypes = [_VP, _VP]
        L.swc_get_stream.restype = _VP
        L.swc_get_stream.argtypes = [_VP]
        L.swc_analyze.argtypes = [_VP, _I] + [_VP] * 6 + [_I] + [_VP] * 2 + [_I] + [_VP] * 3
        L.swc_factor.argtypes = [_VP, _VP, _I, _I, ctypes.POINTER(_I)]
        L.swc_get_L.argtypes = [_VP, _VP, _I]
        L.swc_device_L.restype = _VP
        L.swc_device_L.argtypes = [_VP]
        L.swc_sizes.argtypes = [_VP, _VP]
        L.swc_profile.argtypes = [_VP, _VP, _I, _I, ctypes.POINTER(_I), _VP, _VP, _VP, _VP]
        L.swc_solve.argtypes = [_VP, _VP, _VP, _I, _I]
        L.swc_solve_noalloc.argtypes = [_VP, _VP, _VP, _I]
        L.swc_refine.argtypes = [_VP, _VP, _VP, _I, _I, ctypes.c_double, _I, _VP,
                                 ctypes.POINTER(_I), ctypes.POINTER(_I)]
        L.swc_plan_stats.argtypes = [_I] + [_VP] * 6 + [_I] + [_VP] * 2 + [_I, _VP]
        L.swc_set_plan.argtypes = [_VP, _I]
        L.swc_set_wait_budget.argtypes = [_VP, ctypes.c_longlong]
        L.swc_read_mtx.argtypes = [ctypes.c_char_p, ctypes.POINTER(_I),
                                   ctypes.POINTER(ctypes.POINTER(_I)),
                                   ctypes.POINTER(ctypes.POINTER(_I)),
                                   ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        L.swc_free.restype = None
        L.swc_free.argtypes = [_VP]
        L.swc_write_mtx.argtypes = [ctypes.c_char_p, _I, _VP, _VP, _VP]
        L.swc_read_perm.argtypes = [ctypes.c_char_p, _I, _VP]
        L.swc_write_perm.argtypes = [ctypes.c_char_p, _I, _VP]
        L.swc_order_nd.argtypes = [_I, _VP, _VP, _I, _VP]
        L.swc_layout_sizes.argtypes = [_I] + [_VP] * 3 + [_I, _VP]
        L.swc_layout.argtypes = [_I] + [_VP] * 3 + [_I] + [_VP] * 9
        L.swc_logdet.argtypes = [_VP, ctypes.POINTER(ctypes.c_double)]
        L.swc_logdet_grad.argtypes = [_VP, _VP, _I]
        L.swc_solve_grad.argtypes = [_VP, _VP, _VP, _VP, _I]
        L.swc_supernodes.argtypes = [_I, _VP, _VP, _VP, _VP, _I, _VP, ctypes.POINTER(_I)]
        L.swc_batch_analyze.argtypes = [_VP, _I, _VP, _VP, _VP]
        L.swc_batch_autotune.argtypes = [_VP, _VP, _I, _I, ctypes.c_char_p, _VP, _VP]
        L.swc_batch_berr.argtypes = [_VP, _VP, _VP, _I, _VP]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(rc: int):
    if rc != SWC_OK:
        raise SWCError(rc, lib().swc_last_error().decode())


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def sw_cholesky_left_par_05(n, c, r, values, lC, Ls, Li_ptr, lValues, blockSet, supNo,
                            timing, prunePtr, pruneSet, nLevels, levelPtr, levelSet, nPar,
                            parPtr, partition, chunk, threads, super_max, col_max, nodCost):
    """The reference numeric executor's interface; fills ``lValues`` (float64 numpy array of
    L->xsize entries) in place.  Returns 1 on success, 0 on failure (as the reference's
    driver expects, ``examples/sw_choleskyTest01.cpp:240-244``)."""
    L = lib()
    assert lValues.dtype == np.float64 and lValues.flags.c_contiguous
    args = dict(c=_c(c, np.int32), r=_c(r, np.int32), values=_c(values, np.float64),
                lC=_c(lC, np.uint64), Ls=_c(Ls, np.int32), Li_ptr=_c(Li_ptr, np.uint64),
                blockSet=_c(blockSet, np.int32), prunePtr=_c(prunePtr, np.int32),
                pruneSet=_c(pruneSet, np.int32), levelPtr=_c(levelPtr, np.int32),
                parPtr=_c(parPtr, np.int32), partition=_c(partition, np.int32))
    return L.sw_cholesky_left_par_05(
        int(n), _p(args["c"]), _p(args["r"]), _p(args["values"]), _p(args["lC"]),
        _p(args["Ls"]), _p(args["Li_ptr"]), _p(lValues), _p(args["blockSet"]), int(supNo),
        _p(timing), _p(args["prunePtr"]), _p(args["pruneSet"]), int(nLevels),
        _p(args["levelPtr"]), _p(levelSet), int(nPar), _p(args["parPtr"]),
        _p(args["partition"]), int(chunk), int(threads), int(super_max), int(col_max),
        _p(nodCost))


def last_info() -> int:
    return int(lib().swc_last_info())


def layout(n, c, r, blockSet):
    """BCSC layout of a supernode partition: dict with lC, Ls, Li_ptr, sparent, prunePtr,
    pruneSet, levelPtr, parPtr, partition, xsize."""
    L = lib()
    c = _c(c, np.int32)
    r = _c(r, np.int32)
    bs = _c(blockSet, np.int32)
    ns = bs.size - 1
    sz = np.zeros(4, np.int64)
    _check(L.swc_layout_sizes(int(n), _p(c), _p(r), _p(bs), ns, _p(sz)))
    nls, nprune, xsize, nlev = (int(v) for v in sz)
    out = dict(lC=np.zeros(n + 1, np.uint64), Ls=np.zeros(nls, np.int32),
               Li_ptr=np.zeros(n + 1, np.uint64), sparent=np.zeros(ns, np.int32),
               prunePtr=np.zeros(ns + 1, np.int32), pruneSet=np.zeros(nprune, np.int32),
               levelPtr=np.zeros(nlev + 1, np.int32), parPtr=np.zeros(ns + 1, np.int32),
               partition=np.zeros(ns, np.int32))
    _check(L.swc_layout(int(n), _p(c), _p(r), _p(bs), ns, *[_p(out[k]) for k in (
        "lC", "Ls", "Li_ptr", "sparent", "prunePtr", "pruneSet", "levelPtr", "parPtr",
        "partition")]))
    out["xsize"] = xsize
    return out


def supernodes(n, c, r, max_width: int = 1 << 30, nrelax=None, zrelax=None):
    """Supernode partition (blockSet) of an ordered lower CSC pattern: elimination tree,
    column counts and relaxed chains (the reference's nrelax / zrelax by default)."""
    c = _c(c, np.int32)
    r = _c(r, np.int32)
    nr = None if nrelax is None else _c(nrelax, np.int32)
    zr = None if zrelax is None else _c(zrelax, np.float64)
    bs = np.zeros(int(n) + 1, np.int32)
    ns = ctypes.c_int(0)
    _check(lib().swc_supernodes(int(n), _p(c), _p(r), _p(nr), _p(zr), int(max_width), _p(bs),
                                ctypes.byref(ns)))
    return bs[: ns.value + 1].copy()


class MtxMatrix:
    """Lower triangle of a symmetric matrix in CSC form (``n``, ``indptr``, ``indices``,
    ``data``), as ``read_mtx`` returns it."""

    def __init__(self, n, indptr, indices, data):
        self.n = int(n)
        self.indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        self.indices = np.ascontiguousarray(indices, dtype=np.int32)
        self.data = np.ascontiguousarray(data, dtype=np.float64)


def read_mtx(path: str) -> MtxMatrix:
    """Reads a Matrix Market coordinate file (see ``swc_read_mtx``): the lower triangle,
    rows sorted, diagonal present in every column.  Raises SWCError on a malformed file."""
    L = lib()
    n = _I(0)
    c = ctypes.POINTER(_I)()
    r = ctypes.POINTER(_I)()
    v = ctypes.POINTER(ctypes.c_double)()
    _check(L.swc_read_mtx(os.fsencode(path), ctypes.byref(n), ctypes.byref(c), ctypes.byref(r),
                          ctypes.byref(v)))
    try:
        nn = int(n.value)
        indptr = np.ctypeslib.as_array(c, shape=(nn + 1,)).copy()
        nnz = int(indptr[-1])
        indices = np.ctypeslib.as_array(r, shape=(max(nnz, 1),))[:nnz].copy()
        data = np.ctypeslib.as_array(v, shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        for p in (c, r, v):
            L.swc_free(ctypes.cast(p, _VP))
    return MtxMatrix(nn, indptr, indices, data)


def write_mtx(path: str, n, indptr, indices, data):
    """Writes a lower CSC matrix as a symmetric Matrix Market coordinate file."""
    c, r, v = _c(indptr, np.int32), _c(indices, np.int32), _c(data, np.float64)
    _check(lib().swc_write_mtx(os.fsencode(path), int(n), _p(c), _p(r), _p(v)))


def read_perm(path: str, n: int) -> np.ndarray:
    """Reads a permutation file of n native size_t values (checked to be a permutation)."""
    out = np.zeros(int(n), np.uint64)
    _check(lib().swc_read_perm(os.fsencode(path), int(n), _p(out)))
    return out.astype(np.int64)


def write_perm(path: str, perm):
    """Writes perm (new position k holds original index perm[k]) as n native size_t."""
    p = _c(perm, np.uint64)
    _check(lib().swc_write_perm(os.fsencode(path), int(p.size), _p(p)))


def order_nd(n, indptr, indices, leaf: int = 0) -> np.ndarray:
    """Nested-dissection fill-reducing permutation of a sparse symmetric pattern (lower or
    full CSC); perm[k] = original index at new position k."""
    c, r = _c(indptr, np.int32), _c(indices, np.int32)
    out = np.zeros(int(n), np.uint64)
    _check(lib().swc_order_nd(int(n), _p(c), _p(r), int(leaf), _p(out)))
    return out.astype(np.int64)


PLAN_FIELDS = ("levels", "launches", "small", "tiled", "update_tiles", "update_pairs",
               "trsm_tiles", "syrk_tiles")


def plan_stats(n, c, r, lC, Ls, Li_ptr, blockSet, prunePtr, pruneSet, plan: int = 0):
    """Execution plan (candidate ``plan``, as ``Handle.set_plan``) of a structure, computed
    on the host (no GPU needed): counts and the algorithmic flops / bytes per kernel class."""
    st = np.zeros(8 + 2 * len(KERNEL_CLASSES))
    args = [_c(c, np.int32), _c(r, np.int32), _c(lC, np.uint64), _c(Ls, np.int32),
            _c(Li_ptr, np.uint64), _c(blockSet, np.int32), _c(prunePtr, np.int32),
            _c(pruneSet, np.int32)]
    _check(lib().swc_plan_stats(int(n), _p(args[0]), _p(args[1]), _p(args[2]), _p(args[3]),
                                _p(args[4]), _p(args[5]), args[5].size - 1, _p(args[6]),
                                _p(args[7]), int(plan), _p(st)))
    out = {k: int(st[i]) for i, k in enumerate(PLAN_FIELDS)}
    k = len(KERNEL_CLASSES)
    out["flops"] = {name: float(st[8 + i]) for i, name in enumerate(KERNEL_CLASSES)}
    out["bytes"] = {name: float(st[8 + k + i]) for i, name in enumerate(KERNEL_CLASSES)}
    return out


class Handle:
    """A device-resident factorization on one GPU (``swc_create`` ... ``swc_destroy``)."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = ctypes.c_void_p()
        _check(self._lib.swc_create(ctypes.byref(h), int(device)))
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.swc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        """cudaStream_t of the handle, as an integer (for torch.cuda.ExternalStream)."""
        return int(self._lib.swc_get_stream(self._h) or 0)

    def set_stream(self, stream_ptr: int | None):
        _check(self._lib.swc_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)))

    def analyze(self, n, c, r, lC, Ls, Li_ptr, blockSet, prunePtr, pruneSet,
                levelPtr=None, parPtr=None, partition=None):
        self._keep = [_c(c, np.int32), _c(r, np.int32), _c(lC, np.uint64), _c(Ls, np.int32),
                      _c(Li_ptr, np.uint64), _c(blockSet, np.int32), _c(prunePtr, np.int32),
                      _c(pruneSet, np.int32)]
        c, r, lC, Ls, Li_ptr, bs, pp, ps = self._keep
        sched = [None, None, None]
        nlev = 0
        if levelPtr is not None:
            sched = [_c(levelPtr, np.int32), _c(parPtr, np.int32), _c(partition, np.int32)]
            nlev = sched[0].size - 1
        _check(self._lib.swc_analyze(self._h, int(n), _p(c), _p(r), _p(lC), _p(Ls), _p(Li_ptr),
                                     _p(bs), bs.size - 1, _p(pp), _p(ps), nlev, _p(sched[0]),
                                     _p(sched[1]), _p(sched[2])))
        self.nnz = int(c[int(n)])
        self._keep = None
        sz = np.zeros(6, np.int64)
        _check(self._lib.swc_sizes(self._h, _p(sz)))
        self.n, self.nsuper, self.xsize, self.launches = (int(v) for v in sz[:4])

    def factor(self, values, mode: int = SWC_MODE_FP64) -> int:
        """Factor with A2 values: a numpy array (host) or a CUDA tensor on this device.
        Returns info (0 = success, else failing column + 1); raises on other errors."""
        on_dev = hasattr(values, "data_ptr")
        if not on_dev:
            values = _c(values, np.float64)
        info = ctypes.c_int(0)
        rc = self._lib.swc_factor(self._h, _p(values), 1 if on_dev else 0, int(mode),
                                  ctypes.byref(info))
        if rc not in (SWC_OK, SWC_NOT_SPD):
            _check(rc)
        return int(info.value)

    def transfer_bytes(self):
        """(host-to-device, device-to-host) bytes of the last factor / get_L call."""
        sz = np.zeros(6, np.int64)
        _check(self._lib.swc_sizes(self._h, _p(sz)))
        return int(sz[4]), int(sz[5])

    def profile(self, values, mode: int = SWC_MODE_FP64):
        """One factorization with per-kernel-class event timing.  Returns a dict
        class -> (launches, ms, algorithmic flops, algorithmic bytes)."""
        on_dev = hasattr(values, "data_ptr")
        if not on_dev:
            values = _c(values, np.float64)
        k = len(KERNEL_CLASSES)
        la = np.zeros(k, np.int32)
        ms, fl, by = np.zeros(k), np.zeros(k), np.zeros(k)
        info = ctypes.c_int(0)
        rc = self._lib.swc_profile(self._h, _p(values), 1 if on_dev else 0, int(mode),
                                   ctypes.byref(info), _p(la), _p(ms), _p(fl), _p(by))
        if rc not in (SWC_OK, SWC_NOT_SPD):
            _check(rc)
        return {name: (int(la[i]), float(ms[i]), float(fl[i]), float(by[i]))
                for i, name in enumerate(KERNEL_CLASSES)}

    def solve(self, b, out=None):
        """x = (L L^T)^{-1} b in the factor's ordering; b is (n,) or (n, nrhs) numpy, or a
        CUDA tensor (column-major for several right-hand sides: shape (nrhs, n))."""
        on_dev = hasattr(b, "data_ptr")
        if on_dev:
            nrhs = 1 if b.dim() == 1 else b.shape[0]
            x = out if out is not None else b.clone()
        else:
            b = np.asarray(b, np.float64)
            nrhs = 1 if b.ndim == 1 else b.shape[1]
            b = np.asfortranarray(b)
            x = np.zeros_like(b, order="F")
        _check(self._lib.swc_solve(self._h, _p(b), _p(x), int(nrhs), 1 if on_dev else 0))
        return x

    def refine(self, b, tol: float = 1e-14, maxit: int = 30, out=None):
        """Refined solve (see swc_refine).  Returns (x, berr per rhs, iterations, method)."""
        on_dev = hasattr(b, "data_ptr")
        if on_dev:
            nrhs = 1 if b.dim() == 1 else b.shape[0]
            x = out if out is not None else b.clone()
        else:
            b = np.asarray(b, np.float64)
            nrhs = 1 if b.ndim == 1 else b.shape[1]
            b = np.asfortranarray(b)
            x = out if out is not None else np.zeros_like(b, order="F")
        berr = np.zeros(nrhs)
        it, meth = ctypes.c_int(0), ctypes.c_int(0)
        _check(self._lib.swc_refine(self._h, _p(b), _p(x), int(nrhs), 1 if on_dev else 0,
                                    float(tol), int(maxit), _p(berr), ctypes.byref(it),
                                    ctypes.byref(meth)))
        return x, berr, int(it.value), int(meth.value)

    def set_plan(self, plan: int):
        """Execution-plan candidate for the next analyze / batch_analyze (0 default, 1 larger
        persistent supernodes, 2 no persistent walk, 3 smaller small class, 4 dense steps
        as one dataflow launch per level, 5 FP64 trailing SYRK steps in split-TF32 mode, 6 and
        7 tile-owner descendant updates in split-TF32 mode, staged by TMA or cp.async)."""
        _check(self._lib.swc_set_plan(self._h, int(plan)))

    def set_wait_budget(self, polls: int = -1):
        """Poll budget of the device-side waits (persistent walks, chained solve blocks);
        a wait that runs out makes the call fail with SWC_TIMEOUT.  -1: the default."""
        _check(self._lib.swc_set_wait_budget(self._h, int(polls)))

    def batch_analyze(self, mats):
        """Analyse independent ordered matrices (objects with n, indptr, indices: lower CSC
        of P A P^T) as one block-diagonal batch.  Afterwards factor / solve / refine take
        the matrices' values and vectors concatenated in this order."""
        nn = np.array([int(m.n) for m in mats], np.int32)
        c = np.concatenate([np.asarray(m.indptr, np.int32) for m in mats])
        r = np.concatenate([np.asarray(m.indices, np.int32) for m in mats])
        _check(self._lib.swc_batch_analyze(self._h, int(nn.size), _p(nn), _p(c), _p(r)))
        self.nnz = int(sum(int(m.indptr[-1]) for m in mats))
        self.batch_n = nn
        self.batch_offsets = np.concatenate([[0], np.cumsum(nn.astype(np.int64))])
        sz = np.zeros(6, np.int64)
        _check(self._lib.swc_sizes(self._h, _p(sz)))
        self.n, self.nsuper, self.xsize, self.launches = (int(v) for v in sz[:4])

    def batch_autotune(self, values, mode: int = SWC_MODE_FP64, cache_path: str | None = None):
        """Times the supernode-grouping and plan candidates on these values and keeps the
        fastest.  Returns ((partition, plan), best milliseconds per batch factorization)."""
        on_dev = hasattr(values, "data_ptr")
        if not on_dev:
            values = _c(values, np.float64)
        choice = np.zeros(2, np.int32)
        best = np.zeros(1)
        _check(self._lib.swc_batch_autotune(self._h, _p(values), 1 if on_dev else 0, int(mode),
                                            cache_path.encode() if cache_path else None,
                                            _p(choice), _p(best)))
        self._refresh_sizes()
        return (int(choice[0]), int(choice[1])), float(best[0])

    def _refresh_sizes(self):
        sz = np.zeros(6, np.int64)
        _check(self._lib.swc_sizes(self._h, _p(sz)))
        self.n, self.nsuper, self.xsize, self.launches = (int(v) for v in sz[:4])

    def batch_berr(self, b, x):
        """Backward error of every matrix of the batch for concatenated b and x."""
        on_dev = hasattr(b, "data_ptr")
        if not on_dev:
            b, x = _c(b, np.float64), _c(x, np.float64)
        out = np.zeros(self.batch_n.size)
        _check(self._lib.swc_batch_berr(self._h, _p(b), _p(x), 1 if on_dev else 0, _p(out)))
        return out

    def logdet(self) -> float:
        """log det A of the current factor."""
        v = ctypes.c_double(0.0)
        _check(self._lib.swc_logdet(self._h, ctypes.byref(v)))
        return float(v.value)

    def logdet_grad(self, out=None):
        """d log det A / d values (one entry per stored nonzero of A2)."""
        if out is None:
            out = np.zeros(self.nnz, np.float64)
        _check(self._lib.swc_logdet_grad(self._h, _p(out), 1 if hasattr(out, "data_ptr") else 0))
        return out

    def solve_grad(self, x, lam, out=None):
        """d f / d values for f(x), x = A^{-1} b, given lam = A^{-1} df/dx."""
        on_dev = hasattr(x, "data_ptr")
        if not on_dev:
            x, lam = _c(x, np.float64), _c(lam, np.float64)
        if out is None:
            if on_dev:
                import torch
                out = torch.empty(self.nnz, dtype=torch.float64, device=x.device)
            else:
                out = np.zeros(self.nnz, np.float64)
        _check(self._lib.swc_solve_grad(self._h, _p(x), _p(lam), _p(out), 1 if on_dev else 0))
        return out

    def get_L(self, out=None):
        """L in the reference layout: into ``out`` (numpy or CUDA tensor) or a new numpy array."""
        if out is None:
            out = np.zeros(self.xsize, np.float64)
        _check(self._lib.swc_get_L(self._h, _p(out), 1 if hasattr(out, "data_ptr") else 0))
        return out

    def device_L_ptr(self) -> int:
        return int(self._lib.swc_device_L(self._h) or 0)
