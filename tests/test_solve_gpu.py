"""GPU supernodal solves and FP64 iterative refinement against the oracle's solve.

Tolerances: solve results within 1e-12 (relative, max norm) of the oracle's solve with the
same factor; backward error ||b - A x||_inf / (||A||_inf ||x||_inf) <= 1e-14 after
refinement."""
import numpy as np
import pytest

from conftest import load_small, load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def handle_for(n, A2p, A2i, A2x, lC, Ls, Li_ptr, super_, prunePtr, pruneSet):
    h = swc.Handle(0)
    h.analyze(n, A2p, A2i, lC, Ls, Li_ptr, super_, prunePtr, pruneSet)
    assert h.factor(A2x) == 0
    return h


@pytest.mark.parametrize("name", ["grid2d_20", "grid3d_8", "stencil27_4", "grid2d_100"])
def test_solve_matches_oracle(cuda_ok, name):
    g = load_small(name)
    n = int(g["n"])
    h = handle_for(n, g["A2p"], g["A2i"], g["A2x"], g["lC"], g["Ls"], g["Li_ptr"], g["super"],
                   g["prunePtr"], g["pruneSet"])
    L = h.get_L()
    rng = np.random.default_rng(1)
    B = rng.standard_normal((n, 3))
    X = h.solve(B)
    Xo = O.oracle_solve(n, g["lC"], g["Ls"], g["Li_ptr"], L, g["super"], B)
    assert np.abs(X - Xo).max() <= 1e-12 * np.abs(Xo).max()


@pytest.mark.parametrize("name", ["grid3d_24", "stencil27_12"])
def test_refine_reaches_fp64_backward_error(cuda_ok, name):
    gs = load_sym(name)
    A, _, _ = W.build(name)
    P = W.assemble(A, gs["perm"], gs["super"])
    h = handle_for(P.n, P.A2p, P.A2i, P.A2x, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr,
                   P.pruneSet)
    b = np.random.default_rng(0).standard_normal(P.n)
    x, berr, iters, method = h.refine(b, tol=1e-15, maxit=5)
    r = O.oracle_symv(P.n, P.A2p, P.A2i, P.A2x, x) - b
    Afull = A.to_scipy_full()
    anorm = abs(Afull).sum(axis=1).max()
    assert np.abs(r).max() / (anorm * np.abs(x).max()) <= 1e-14
    assert berr[0] <= 1e-14


def test_solve_device_tensor(cuda_ok):
    import torch
    g = load_small("grid3d_8")
    n = int(g["n"])
    h = handle_for(n, g["A2p"], g["A2i"], g["A2x"], g["lC"], g["Ls"], g["Li_ptr"], g["super"],
                   g["prunePtr"], g["pruneSet"])
    b = torch.from_numpy(g["b"]).cuda()
    x = h.solve(b)
    xo = O.oracle_solve(n, g["lC"], g["Ls"], g["Li_ptr"], g["L"], g["super"], g["b"])
    assert np.abs(x.cpu().numpy() - xo).max() <= 1e-12 * np.abs(xo).max()
