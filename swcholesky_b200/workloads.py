"""Named workloads and their assembly into the numeric-phase inputs.

Each workload is a seeded synthetic SPD matrix plus the geometric nested-dissection user
permutation for it.  They stand in for the reference's SuiteSparse inputs, which it does
not ship:

=============  ===========================================================================
grid2d_100     2D 5-point Laplacian, 100 x 100, Dirichlet (n = 10,000)
grid3d_60      3D 7-point Laplacian, 60^3, diagonal shift 1e-3 (n = 216,000)
stencil27_40   3-dof 27-point weighted stencil, 40^3 (n = 192,000), shift for cond ~ 1e6
stencil27_40c10  the same operator with the shift for cond ~ 1e10
gmrf_500       GMRF precision 0.1 I + weighted 5-point Laplacian, 500 x 500 (n = 250,000)
batch256       256 weighted 5-point grids, sides uniform in [30, 200] (n 900 .. 40,000),
               log-normal(0.5) conductances, shift 1e-4 (``batch_matrices``)
grid2d_20, grid3d_8, stencil27_4   small cases of the same families, for tests
=============  ===========================================================================

``assemble(A, perm, super)`` turns a matrix, the final permutation and a supernode
partition (what the reference's symbolic phase produces) into every array the numeric
entry point takes, using the library's layout builder.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import matrices as M

__all__ = ["build", "assemble", "assemble_own", "batch_matrices", "Problem", "cond_shift"]


def cond_shift(L: M.LowerCSC, cond: float) -> float:
    """Diagonal shift giving cond(L + shift*I) = cond (see ``matrices.cond_shift``)."""
    return M.cond_shift(L, cond)


def build(name: str):
    """Returns (A as LowerCSC in the original order, user permutation, meta dict)."""
    return M.workload_matrix(name)


@dataclass
class Problem:
    n: int
    A2p: np.ndarray
    A2i: np.ndarray
    A2x: np.ndarray
    super: np.ndarray
    lC: np.ndarray
    Ls: np.ndarray
    Li_ptr: np.ndarray
    sparent: np.ndarray
    prunePtr: np.ndarray
    pruneSet: np.ndarray
    levelPtr: np.ndarray
    parPtr: np.ndarray
    partition: np.ndarray
    xsize: int
    perm: np.ndarray

    @property
    def nsuper(self) -> int:
        return int(self.super.size - 1)


def assemble(A: M.LowerCSC, perm, super_) -> Problem:
    from . import layout
    perm = np.asarray(perm)
    A2 = M.permute_lower(A, perm)
    lay = layout(A2.n, A2.indptr, A2.indices, super_)
    return Problem(n=A2.n, A2p=A2.indptr, A2i=A2.indices, A2x=A2.data,
                   super=np.ascontiguousarray(super_, np.int32), lC=lay["lC"], Ls=lay["Ls"],
                   Li_ptr=lay["Li_ptr"], sparent=lay["sparent"], prunePtr=lay["prunePtr"],
                   pruneSet=lay["pruneSet"], levelPtr=lay["levelPtr"], parPtr=lay["parPtr"],
                   partition=lay["partition"], xsize=int(lay["xsize"]), perm=perm)


def assemble_own(A: M.LowerCSC, perm, max_width: int = 1 << 30, nrelax=None,
                 zrelax=None) -> Problem:
    """As ``assemble``, with the library's own supernode partition (elimination tree,
    column counts, relaxed chains) instead of one from the reference's symbolic phase."""
    from . import supernodes
    perm = np.asarray(perm)
    A2 = M.permute_lower(A, perm)
    super_ = supernodes(A2.n, A2.indptr, A2.indices, max_width=max_width, nrelax=nrelax,
                        zrelax=zrelax)
    return assemble(A, perm, super_)


def batch_sources(count: int = 256, seed: int = 0, lo: int = 30, hi: int = 200,
                  sigma: float = 0.5, shift: float = 1e-4):
    """Independent SPD matrices of uneven size for the batched path: weighted 5-point grids
    with sides drawn uniformly from [lo, hi], log-normal(sigma) edge conductances and a
    diagonal shift.  Returns [(A in natural order, nested-dissection perm)] and the sides."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, count)
    out = []
    for k, s in enumerate(sides):
        s = int(s)
        A = M.weighted_grid_2d(s, sigma=sigma, shift=shift, seed=seed * 100003 + k + 1)
        out.append((A, M.nested_dissection((s, s))))
    return out, sides


def batch_matrices(count: int = 256, seed: int = 0, lo: int = 30, hi: int = 200,
                   sigma: float = 0.5, shift: float = 1e-4):
    """The matrices of ``batch_sources``, each ordered (lower CSC of P A P^T)."""
    src, sides = batch_sources(count, seed, lo, hi, sigma, shift)
    return [M.permute_lower(A, perm) for A, perm in src], sides
