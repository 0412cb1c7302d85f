"""Task lists of the supernodal solves, checked on the host (no GPU).

The solves walk the supernodal elimination tree level by level.  The forward solve follows
the reference's blockedLsolve (triangularSolve/Triangular_BCSC.h:14-48) in gather form.
The library's plan check requires:
  * every supernode solved exactly once, in a level after its children's: by a warp, by a
    CTA, or (tiled class) by one chained block per 64 columns, forward in increasing and
    backward in decreasing block order;
  * every off-diagonal row of a CTA-solved supernode in exactly one forward contribution
    task (32- or 128-row tasks, aligned to the first off-diagonal row);
  * every 16-column group of such a supernode in exactly one backward gather task;
  * each column's contribution list naming exactly the contributions of the rows equal to
    it, so the forward solve sums each contribution once.
swc_plan_stats raises on the first violation."""
import pytest

from conftest import load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import workloads as W


def problem(name):
    gs = load_sym(name)
    A, _, _ = W.build(name)
    return W.assemble(A, gs["perm"], gs["super"])


@pytest.mark.parametrize("name", ["grid2d_100", "grid3d_24", "stencil27_12", "gmrf_500",
                                  "grid3d_60"])
def test_solve_plan_covers_every_row_and_column_once(name):
    P = problem(name)
    args = (P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    for plan in ([0, 3] if name != "grid3d_60" else [0]):   # default and larger small class
        stats = swc.plan_stats(*args, plan=plan)              # raises on a violation
        assert stats["levels"] >= 1


def test_solve_plan_on_own_partition():
    """A partition from the library's own supernode builder (not the reference's)."""
    A, perm, _ = W.build("grid3d_24")
    P = W.assemble_own(A, perm)
    swc.plan_stats(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
