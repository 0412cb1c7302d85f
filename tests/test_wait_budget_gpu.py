"""Bounded device-side waits, driven to run out through the handle's poll budget.

Every wait of the library's kernels on another CTA's result is bounded: the persistent
walks of the factorization (a supernode waiting for the descendants in its update list)
and the chained diagonal blocks of the triangular solves (a block waiting for the block
before it).  With a budget of 0 polls a wait gives up unless its flag is already set, the
kernels return with the timeout recorded in the status words, and the call fails with
SWC_TIMEOUT; the handle stays usable and the next call with the default budget is correct.
No GPU fault, trap or hang is involved: the wait just stops polling."""
import numpy as np
import pytest

from conftest import load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grid3d_24():
    gs = load_sym("grid3d_24")
    A, _, _ = W.build("grid3d_24")
    return W.assemble(A, gs["perm"], gs["super"])


def _handle(P):
    h = swc.Handle(0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    return h


def test_factor_walk_timeout_then_recovers(cuda_ok, grid3d_24):
    P = grid3d_24
    plan = swc.plan_stats(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr,
                          P.pruneSet)
    assert plan["small"] > 0     # the persistent walks have supernodes that wait
    h = _handle(P)
    h.set_wait_budget(0)
    timeouts = 0
    for _ in range(3):           # a wait whose flag happens to be set already does not fail
        try:
            h.factor(P.A2x)
        except swc.SWCError as e:
            assert e.code == swc.SWC_TIMEOUT, str(e)
            assert "waited longer than its budget" in str(e)
            timeouts += 1
    assert timeouts > 0
    h.set_wait_budget(-1)
    assert h.factor(P.A2x) == 0
    Lo, ok, _ = O.oracle_factor(P.n, P.A2p, P.A2i, P.A2x, P.lC, P.Ls, P.Li_ptr, P.super,
                                P.prunePtr, P.pruneSet, P.levelPtr, P.parPtr, P.partition,
                                P.xsize)
    assert ok == 1
    L = h.get_L()
    assert np.abs(L - Lo).max() <= 1e-12 * np.abs(Lo).max()


def test_solve_chain_timeout_then_recovers(cuda_ok, grid3d_24):
    P = grid3d_24
    plan = swc.plan_stats(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr,
                          P.pruneSet)
    assert plan["tiled"] > 0     # wide supernodes: chained blocks in both solves
    h = _handle(P)
    assert h.factor(P.A2x) == 0
    b = np.random.default_rng(5).standard_normal(P.n)
    x_ok = h.solve(b)
    h.set_wait_budget(0)
    timeouts = 0
    for _ in range(3):
        try:
            h.solve(b)
        except swc.SWCError as e:
            assert e.code == swc.SWC_TIMEOUT, str(e)
            assert "triangular solve" in str(e)
            timeouts += 1
    assert timeouts > 0
    h.set_wait_budget(-1)
    x = h.solve(b)
    assert np.abs(x - x_ok).max() <= 1e-12 * np.abs(x_ok).max()
