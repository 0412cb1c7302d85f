"""Execution-plan candidate 4: the dense factorization of each level's tiled-class
supernodes as one persistent dataflow launch (diagonal blocks, TRSM tiles and grouped
trailing updates as tasks with per-tile version counters) instead of three launches per
64-column step.

CPU: the plan builder replays every wait of the task list in list order and rejects an
order in which a task waits for a later one (the walk could stall), so building the plan
for the workloads' structures checks the order; the algorithmic work is the same as the
default plan's.  GPU: the dataflow factor against the oracle (FP64, tolerance 1e-12 of
max |L|, as the default plan) and a mixed-precision factor refined to 1e-14."""
import numpy as np
import pytest

from conftest import load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import workloads as W
from oracle import oracle as O

DATAFLOW = 4
RTOL_L = 1e-12


def problem(name):
    gs = load_sym(name)
    A, _, _ = W.build(name)
    return A, W.assemble(A, gs["perm"], gs["super"])


@pytest.mark.parametrize("name", ["grid3d_24", "stencil27_12", "gmrf_500", "grid2d_100"])
def test_dataflow_plan_order_and_work(name):
    _, P = problem(name)
    args = (P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    base = swc.plan_stats(*args)
    df = swc.plan_stats(*args, plan=DATAFLOW)       # raises if the order could stall
    assert df["tiled"] == base["tiled"]
    if base["tiled"]:
        assert df["launches"] < base["launches"]
    # the dense class carries the trailing updates in the dataflow plan: same total work
    fb, fd = base["flops"], df["flops"]
    assert fd["syrk"] == 0.0
    assert fd["panel"] == pytest.approx(fb["panel"] + fb["syrk"], rel=1e-12)
    assert fd["update"] == fb["update"]


@pytest.mark.parametrize("max_width", [1 << 30, 200, 130, 100, 65, 64, 40])
def test_dataflow_plan_own_partition(max_width):
    """Library partitions of a 3D grid with supernode width caps: the tiled supernodes' last
    column blocks are 1 to 60 columns wide or full (width mod 64 over the caps: 0, 1, 2, 4,
    8, 16, 24, 30, 32, 36, 40, 44, 55-60), and narrow tiled supernodes have many rows."""
    A, perm, _ = W.build("grid3d_24")
    P = W.assemble_own(A, perm, max_width=max_width)
    w = np.diff(P.super)
    assert w.max() <= max_width
    args = (P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    base = swc.plan_stats(*args)
    df = swc.plan_stats(*args, plan=DATAFLOW)       # raises if the order could stall
    assert df["flops"]["panel"] == pytest.approx(base["flops"]["panel"] + base["flops"]["syrk"],
                                                 rel=1e-12)


def test_unknown_plan_rejected():
    _, P = problem("grid2d_100")
    with pytest.raises(swc.SWCError):
        swc.plan_stats(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr,
                       P.pruneSet, plan=99)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["grid3d_24", "stencil27_12"])
def test_dataflow_factor_matches_oracle(cuda_ok, name):
    A, P = problem(name)
    Lo, ok, _ = O.oracle_factor(P.n, P.A2p, P.A2i, P.A2x, P.lC, P.Ls, P.Li_ptr, P.super,
                                P.prunePtr, P.pruneSet, P.levelPtr, P.parPtr, P.partition,
                                P.xsize)
    assert ok == 1
    h = swc.Handle(0)
    h.set_plan(DATAFLOW)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h.factor(P.A2x) == 0
    L = h.get_L()
    assert float(np.abs(L - Lo).max() / np.abs(Lo).max()) <= RTOL_L
    assert np.all(L[Lo == 0.0] == 0.0)
    assert h.factor(P.A2x) == 0                      # graph replay, same result
    assert np.array_equal(h.get_L(), L)
    # mixed precision through the same plan, refined in FP64
    assert h.factor(P.A2x, swc.SWC_MODE_MIXED_TF32X3) == 0
    b = np.random.default_rng(1).standard_normal(P.n)
    x, berr, _, _ = h.refine(b, tol=1e-14, maxit=30)
    assert berr.max() <= 1e-14


@pytest.mark.gpu
def test_dataflow_not_spd_reports_column(cuda_ok):
    """A non-positive pivot inside a tiled supernode is reported as with the default plan."""
    _, P = problem("grid3d_24")
    h = swc.Handle(0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    col = int(P.super[-2])                            # first column of the root supernode
    vals = P.A2x.copy()
    p = int(P.A2p[col])
    assert P.A2i[p] == col
    vals[p] = -1.0
    info_default = h.factor(vals)
    h4 = swc.Handle(0)
    h4.set_plan(DATAFLOW)
    h4.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h4.factor(vals) == info_default > 0
