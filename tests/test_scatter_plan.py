"""Tables of the mixed modes' right-looking updates, checked on the host (no GPU).

A descendant's contribution C = B B^T is formed as dense 128x128 tiles and added to L by
FP64 atomic adds through a per-column table (the target's first entry) and per-row
relative indices (the reference's relative-index scatter, cholesky/sw_parallel_PB_Cholesky_05_check.c:
the row map of the update into the target's rows).  The library's plan check compares
every scattered entry's address with a direct lookup in the target's row list, and checks
that each descendant's lower triangle is covered once per column of K (also when the plan
cuts K into 256- or 128-column tiles), that every tile runs in the level after its
descendant's, and that the dense steps' trailing-update tiles give every column block each
earlier column block exactly once, each step's next-column tiles (launched on the chain's
stream) ahead of its grouped ones (launched beside the following steps)."""
import pytest

from conftest import load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import workloads as W

PLANS = [0, 5, 8, 9]   # default, FP64 SYRK steps, K cut at 256 and at 128 columns


def problem(name):
    gs = load_sym(name)
    A, _, _ = W.build(name)
    return W.assemble(A, gs["perm"], gs["super"])


@pytest.mark.parametrize("name", ["grid3d_24", "stencil27_12", "gmrf_500", "grid3d_60"])
def test_scatter_tables_match_direct_lookup(name):
    P = problem(name)
    args = (P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    plans = PLANS if name != "grid3d_60" else [0, 9]
    stats = [swc.plan_stats(*args, plan=p) for p in plans]   # raises on a violation
    # cutting K changes the number of tiles, not the plan's work or levels
    for s in stats[1:]:
        assert s["levels"] == stats[0]["levels"]
        assert s["flops"] == stats[0]["flops"]
