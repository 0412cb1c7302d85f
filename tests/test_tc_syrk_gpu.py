"""Plan candidate 5: the trailing SYRK steps of the split-TF32 factorization on the tcgen05
tensor cores (swc_tc.cu: kind::tf32 products of the split mirror viewed as 128-row
operands, TMEM accumulators, FP64 tile update).

Checked like the other mixed paths: against the FP64 factor of the same matrix (relative
difference of L above 1e-12, below the split-TF32 bound for the Laplacian and for the
cond ~1e6 stencil) and by FP64 refinement to backward error <= 1e-14; the plan must also
match the default split-TF32 plan closely (both are FP32-class approximations of L)."""
import numpy as np
import pytest

from conftest import load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import workloads as W

pytestmark = pytest.mark.gpu

TC_PLAN = 5


@pytest.mark.parametrize("name,lbound", [("grid3d_24", 1e-5), ("stencil27_12", 1e-2)])
def test_tc_syrk_mixed_factor(cuda_ok, name, lbound):
    gs = load_sym(name)
    A, _, _ = W.build(name)
    P = W.assemble(A, gs["perm"], gs["super"])
    h0 = swc.Handle(0)
    h0.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h0.factor(P.A2x, swc.SWC_MODE_FP64) == 0
    L64 = h0.get_L()
    assert h0.factor(P.A2x, swc.SWC_MODE_MIXED_TF32X3) == 0
    Lmx = h0.get_L()
    h = swc.Handle(0)
    h.set_plan(TC_PLAN)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h.factor(P.A2x, swc.SWC_MODE_MIXED_TF32X3) == 0
    Ltc = h.get_L()
    rel = np.abs(Ltc - L64).max() / np.abs(L64).max()
    assert 1e-12 < rel < lbound, rel
    assert np.abs(Ltc - Lmx).max() / np.abs(L64).max() < lbound
    assert h.factor(P.A2x, swc.SWC_MODE_MIXED_TF32X3) == 0   # graph replay: same result
    assert np.array_equal(h.get_L(), Ltc)
    b = np.random.default_rng(2).standard_normal(P.n)
    x, berr, iters, method = h.refine(b, tol=1e-14, maxit=30)
    assert berr.max() <= 1e-14
    # FP64 mode on the same plan is unchanged (the tcgen05 path is split-TF32 only)
    assert h.factor(P.A2x, swc.SWC_MODE_FP64) == 0
    assert np.abs(h.get_L() - L64).max() <= 1e-12 * np.abs(L64).max()
