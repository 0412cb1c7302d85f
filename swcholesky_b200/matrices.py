"""Synthetic SPD workloads and a geometric nested-dissection ordering for grid problems.

The reference factors SuiteSparse matrices read from Matrix Market files with a METIS
permutation computed elsewhere (``examples/sw_choleskyTest01.cpp:57-82``); neither the
matrices nor the ordering tool ship with it.  These seeded generators produce the
workloads the factorization is measured on, and ``nested_dissection`` produces the user
permutation that the reference's symbolic phase takes as input (``GIVEN``,
``cholesky/sw_LSparsity.h:461-468``).

Every matrix is returned as the LOWER triangle in CSC form with sorted row indices and a
non-empty diagonal in every column, the input format the reference's reader produces
(``common/Util.h:97-176``).  A permutation ``perm`` follows the CHOLMOD convention used by
the reference: new position ``k`` holds original column ``perm[k]``.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

__all__ = [
    "LowerCSC",
    "laplacian_2d",
    "laplacian_3d",
    "weighted_grid_2d",
    "stencil27_3dof",
    "nested_dissection",
    "permute_lower",
    "cond_shift",
    "workload_matrix",
    "random_geometric",
]


class LowerCSC:
    """Lower triangle of a symmetric matrix: int32 ``indptr``/``indices``, float64 ``data``."""

    def __init__(self, n: int, indptr, indices, data):
        self.n = int(n)
        self.indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        self.indices = np.ascontiguousarray(indices, dtype=np.int32)
        self.data = np.ascontiguousarray(data, dtype=np.float64)

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def to_scipy_full(self) -> sp.csc_matrix:
        low = sp.csc_matrix((self.data, self.indices, self.indptr), shape=(self.n, self.n))
        full = low + sp.tril(low, -1).T
        return sp.csc_matrix(full)

    @staticmethod
    def from_scipy(mat) -> "LowerCSC":
        low = sp.csc_matrix(sp.tril(sp.csc_matrix(mat)))
        low.sum_duplicates()
        low.sort_indices()
        return LowerCSC(low.shape[0], low.indptr, low.indices, low.data)


def _grid_index(dims):
    return np.arange(int(np.prod(dims))).reshape(dims[::-1]).transpose()


def _edges(dims, offsets):
    """All (u, v) node pairs of a regular grid for the given neighbour offsets (u < v)."""
    idx = _grid_index(dims)
    us, vs = [], []
    for off in offsets:
        sl_u, sl_v = [], []
        for d, o in enumerate(off):
            if o >= 0:
                sl_u.append(slice(0, dims[d] - o))
                sl_v.append(slice(o, dims[d]))
            else:
                sl_u.append(slice(-o, dims[d]))
                sl_v.append(slice(0, dims[d] + o))
        u = idx[tuple(sl_u)].ravel()
        v = idx[tuple(sl_v)].ravel()
        us.append(u)
        vs.append(v)
    u = np.concatenate(us)
    v = np.concatenate(vs)
    lo = np.minimum(u, v)
    hi = np.maximum(u, v)
    return lo, hi


def _assemble(n, diag, lo, hi, w):
    rows = np.concatenate([np.arange(n), hi])
    cols = np.concatenate([np.arange(n), lo])
    vals = np.concatenate([diag, w])
    low = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    low.sum_duplicates()
    low.sort_indices()
    return LowerCSC(n, low.indptr, low.indices, low.data)


def laplacian_2d(nx: int, ny: int | None = None, shift: float = 0.0) -> LowerCSC:
    """5-point Laplacian on an nx-by-ny grid, Dirichlet boundary: diag 4 + shift, off -1."""
    ny = nx if ny is None else ny
    n = nx * ny
    lo, hi = _edges((nx, ny), [(1, 0), (0, 1)])
    return _assemble(n, np.full(n, 4.0 + shift), lo, hi, np.full(lo.size, -1.0))


def laplacian_3d(k: int, shift: float = 0.0) -> LowerCSC:
    """7-point Laplacian on a k^3 grid, Dirichlet boundary: diag 6 + shift, off -1."""
    n = k ** 3
    lo, hi = _edges((k, k, k), [(1, 0, 0), (0, 1, 0), (0, 0, 1)])
    return _assemble(n, np.full(n, 6.0 + shift), lo, hi, np.full(lo.size, -1.0))


def weighted_grid_2d(nx: int, ny: int | None = None, sigma: float = 0.5,
                     shift: float = 1e-4, seed: int = 0) -> LowerCSC:
    """Weighted 5-point graph Laplacian (log-normal(sigma) edge weights) plus shift*I.

    The graph Laplacian is singular (constants are in its null space); the shift makes the
    matrix SPD with cond(A) = (lambda_max + shift) / shift."""
    ny = nx if ny is None else ny
    n = nx * ny
    rng = np.random.default_rng(seed)
    lo, hi = _edges((nx, ny), [(1, 0), (0, 1)])
    w = np.exp(sigma * rng.standard_normal(lo.size))
    deg = np.zeros(n)
    np.add.at(deg, lo, w)
    np.add.at(deg, hi, w)
    return _assemble(n, deg + shift, lo, hi, -w)


def stencil27_3dof(k: int, sigma: float = 1.0, shift: float = 0.0, seed: int = 0) -> LowerCSC:
    """3-dof-per-node 27-point weighted graph Laplacian on a k^3 grid plus shift*I.

    Each grid edge (i, j) carries a 3x3 SPD coupling B_ij = w_ij * G_ij with w_ij
    log-normal(sigma) and G_ij = Q diag(d) Q^T (Q from a seeded QR, d uniform in [1, 2]).
    The operator is sum_edges (e_i - e_j)(e_i - e_j)^T (x) B_ij + shift*I, which is SPD
    for shift > 0."""
    nn = k ** 3
    n = 3 * nn
    rng = np.random.default_rng(seed)
    offs = [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)
            if (a, b, c) > (0, 0, 0)]
    lo, hi = _edges((k, k, k), offs)
    ne = lo.size
    g = rng.standard_normal((ne, 3, 3))
    q, _ = np.linalg.qr(g)
    d = rng.uniform(1.0, 2.0, size=(ne, 3))
    G = np.einsum("eij,ej,ekj->eik", q, d, q)
    w = np.exp(sigma * rng.standard_normal(ne))
    B = G * w[:, None, None]
    # node diagonal blocks: sum of incident B
    D = np.zeros((nn, 3, 3))
    np.add.at(D, lo, B)
    np.add.at(D, hi, B)
    r_d, c_d = np.meshgrid(np.arange(3), np.arange(3), indexing="ij")
    rows = [(3 * np.arange(nn))[:, None, None] + r_d, (3 * hi)[:, None, None] + r_d]
    cols = [(3 * np.arange(nn))[:, None, None] + c_d, (3 * lo)[:, None, None] + c_d]
    vals = [D, -B]
    rows = np.concatenate([x.ravel() for x in rows])
    cols = np.concatenate([x.ravel() for x in cols])
    vals = np.concatenate([x.ravel() for x in vals])
    keep = rows >= cols
    full = sp.csc_matrix((vals[keep], (rows[keep], cols[keep])), shape=(n, n))
    full = full + sp.identity(n, format="csc") * shift
    return LowerCSC.from_scipy(full)


def nested_dissection(dims, dof: int = 1, leaf: int = 8) -> np.ndarray:
    """Geometric nested dissection of a regular grid (any dimension), separator last.

    A box is split across its longest side by the middle plane of nodes; both halves are
    ordered recursively, then the plane.  One plane separates the 5-, 7- and 27-point
    stencils alike.  Boxes with at most ``leaf`` nodes keep their natural order.  With
    ``dof`` > 1 the dofs of a node stay consecutive.  Returns perm (int64): new position
    k holds original index perm[k]."""
    dims = tuple(int(d) for d in dims)
    idx = _grid_index(dims)
    out = []
    # explicit LIFO work list; a box expands to [left, right, plane], emitted in that order
    work = [("box", tuple((0, d) for d in dims))]
    while work:
        kind, payload = work.pop()
        if kind == "nodes":
            out.append(payload)
            continue
        box = payload
        sizes = [b - a for a, b in box]
        count = int(np.prod(sizes))
        if count == 0:
            continue
        if count <= leaf or max(sizes) < 3:
            sub = idx[tuple(slice(a, b) for a, b in box)]
            out.append(sub.transpose().ravel())
            continue
        d = int(np.argmax(sizes))
        a, b = box[d]
        m = (a + b) // 2
        left = tuple((a, m) if i == d else box[i] for i in range(len(box)))
        right = tuple((m + 1, b) if i == d else box[i] for i in range(len(box)))
        plane = tuple((m, m + 1) if i == d else box[i] for i in range(len(box)))
        plane_nodes = idx[tuple(slice(p, q) for p, q in plane)].transpose().ravel()
        # stack is LIFO: push plane first so it is emitted last
        work.append(("nodes", plane_nodes))
        work.append(("box", right))
        work.append(("box", left))
    node_perm = np.concatenate(out).astype(np.int64)
    if dof == 1:
        return node_perm
    return (dof * node_perm[:, None] + np.arange(dof)[None, :]).ravel().astype(np.int64)


def permute_lower(A: LowerCSC, perm: np.ndarray) -> LowerCSC:
    """Lower triangle of P A P^T with sorted rows, where (P A P^T)[k, l] = A[perm[k], perm[l]]."""
    full = A.to_scipy_full()
    p = np.asarray(perm)
    B = full[p][:, p]
    return LowerCSC.from_scipy(B)


def random_geometric(n: int, dim: int = 3, degree: float = 10.0, sigma: float = 0.5,
                     shift: float = 1e-2, seed: int = 0) -> LowerCSC:
    """SPD matrix of a random geometric graph, a structure with no grid to dissect: n points
    uniform in the unit square (dim 2) or cube (dim 3), joined when closer than the radius
    that gives `degree` neighbours on average; log-normal(sigma) edge weights; the weighted
    graph Laplacian plus shift * I."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    X = rng.random((n, dim))
    vol = np.pi if dim == 2 else 4.0 / 3.0 * np.pi
    radius = (degree / (n * vol)) ** (1.0 / dim)
    pairs = cKDTree(X).query_pairs(radius, output_type="ndarray")
    w = rng.lognormal(0.0, sigma, len(pairs))
    W = sp.coo_matrix((w, (pairs[:, 0], pairs[:, 1])), shape=(n, n))
    W = (W + W.T).tocsc()
    Lap = sp.diags(np.asarray(W.sum(axis=1)).ravel()) - W + shift * sp.identity(n)
    return LowerCSC.from_scipy(Lap)


def cond_shift(L: LowerCSC, cond: float) -> float:
    """Diagonal shift giving cond(L + shift*I) = cond for a singular PSD graph Laplacian L
    (lambda_min = 0), from a Lanczos estimate of lambda_max."""
    import scipy.sparse.linalg as sla
    lmax = float(sla.eigsh(L.to_scipy_full(), k=1, which="LA", return_eigenvectors=False,
                           tol=1e-6)[0])
    return lmax / (cond - 1.0)


def workload_matrix(name: str):
    """A named workload: (A as LowerCSC in the original order, user permutation, meta).

    grid2d_<k>: 2D 5-point Laplacian k x k (Dirichlet); grid3d_<k>: 3D 7-point Laplacian
    k^3 plus 1e-3 I; stencil27_<k>[c10]: 3-dof 27-point weighted stencil k^3 shifted to
    cond ~1e6 (~1e10 with the c10 suffix); gmrf_<k>: 0.1 I + log-normal(0.7) weighted
    5-point Laplacian k x k.  The permutation is the geometric nested dissection of the
    grid.  Depends on numpy and scipy only."""
    if name.startswith("grid2d_"):
        k = int(name.split("_")[1])
        return laplacian_2d(k), nested_dissection((k, k)), dict(kind="laplacian2d", k=k)
    if name.startswith("grid3d_"):
        k = int(name.split("_")[1])
        shift = 1e-3
        return (laplacian_3d(k, shift), nested_dissection((k, k, k)),
                dict(kind="laplacian3d", k=k, shift=shift))
    if name.startswith("stencil27_"):
        tag = name.split("_")[1]
        cond = 1e10 if tag.endswith("c10") else 1e6
        k = int(tag.replace("c10", ""))
        L0 = stencil27_3dof(k, sigma=1.0, shift=0.0, seed=0)
        shift = cond_shift(L0, cond)
        A = stencil27_3dof(k, sigma=1.0, shift=shift, seed=0)
        return A, nested_dissection((k, k, k), dof=3), dict(kind="stencil27x3", k=k,
                                                                 cond=cond, shift=shift)
    if name.startswith("gmrf_"):
        k = int(name.split("_")[1])
        A = weighted_grid_2d(k, sigma=0.7, shift=0.1, seed=0)
        return A, nested_dissection((k, k)), dict(kind="gmrf", k=k, kappa2=0.1)
    raise KeyError(name)
