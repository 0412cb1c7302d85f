"""Mixed-precision factorization (split-TF32 or BF16x3 Schur updates) followed by FP64
refinement.

The mixed factor differs from the FP64 one by FP32-class rounding amplified by the
conditioning (checked: relative difference of L above 1e-12, below 1e-5 for the Laplacian
and below 1e-2 for the cond ~1e6 stencil), and refinement against the FP64 matrix reaches
the FP64 backward error (<= 1e-14)."""
import numpy as np
import pytest

from conftest import load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


MODES = [swc.SWC_MODE_MIXED_TF32X3, swc.SWC_MODE_MIXED_BF16X3]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name,lbound", [("grid3d_24", 1e-5), ("stencil27_12", 1e-2)])
def test_mixed_factor_then_refine(cuda_ok, name, lbound, mode):
    gs = load_sym(name)
    A, _, _ = W.build(name)
    P = W.assemble(A, gs["perm"], gs["super"])
    h = swc.Handle(0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h.factor(P.A2x, swc.SWC_MODE_FP64) == 0
    L64 = h.get_L()
    assert h.factor(P.A2x, mode) == 0
    Lmx = h.get_L()
    rel = np.abs(Lmx - L64).max() / np.abs(L64).max()
    assert 1e-12 < rel < lbound, rel
    # right-looking updates summed by FP64 atomics in no fixed order: reproducible to
    # rounding, far below the mixed-vs-FP64 difference
    assert h.factor(P.A2x, mode) == 0
    rerun = np.abs(h.get_L() - Lmx).max() / np.abs(L64).max()
    assert rerun <= 1e-12 and rerun <= 1e-3 * rel, (rerun, rel)
    rng = np.random.default_rng(0)
    b = rng.standard_normal((P.n, 2))
    x, berr, iters, method = h.refine(b, tol=1e-14, maxit=30)
    assert method in (1, 2) and iters >= 1
    assert berr.max() <= 1e-14
    Afull = A.to_scipy_full()
    anorm = abs(Afull).sum(axis=1).max()
    for k in range(2):
        r = O.oracle_symv(P.n, P.A2p, P.A2i, P.A2x, x[:, k]) - b[:, k]
        assert np.abs(r).max() / (anorm * np.abs(x[:, k]).max()) <= 1e-14


@pytest.mark.parametrize("name,mode", [("stencil27_40", swc.SWC_MODE_MIXED_TF32X3),
                                       ("stencil27_40", swc.SWC_MODE_MIXED_BF16X3),
                                       ("stencil27_40c10", swc.SWC_MODE_MIXED_TF32X3),
                                       ("stencil27_40c10", swc.SWC_MODE_MIXED_BF16X3)])
def test_stencil27_40_eight_rhs(cuda_ok, name, mode):
    """The 3-dof 27-point stencil on 40^3 (n = 192,000) at cond ~1e6 and ~1e10: split-TF32
    or BF16x3 factor, FP64 refinement (CG with the factor as preconditioner when refinement stalls)
    of 8 right-hand sides to backward error <= 1e-12 each; per right-hand side the forward
    difference from the FP64 factor's refined solution stays within cond * 1e-13."""
    import torch
    gs = load_sym("stencil27_40")          # the c10 variant shares the structure
    A, _, meta = W.build(name)
    P = W.assemble(A, gs["perm"], gs["super"])
    h = swc.Handle(0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    v = torch.tensor(P.A2x, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(8)
    b = torch.tensor(rng.standard_normal((8, P.n)), dtype=torch.float64, device="cuda")
    assert h.factor(v, swc.SWC_MODE_FP64) == 0
    x64, berr64, _, _ = h.refine(b, tol=1e-14, maxit=30)
    assert h.factor(v, mode) == 0
    xmx, berr, iters, method = h.refine(b, tol=1e-12, maxit=60)
    assert berr.shape == (8,) and berr.max() <= 1e-12, (berr, iters, method)
    fwd = ((xmx - x64).abs().amax(dim=1) / x64.abs().amax(dim=1)).cpu().numpy()
    assert fwd.max() <= meta["cond"] * 1e-13, fwd


@pytest.mark.parametrize("mode,plan", [(swc.SWC_MODE_MIXED_TF32X3, 0),
                                       (swc.SWC_MODE_MIXED_TF32X3, 5),
                                       (swc.SWC_MODE_MIXED_TF32X3, 6),
                                       (swc.SWC_MODE_MIXED_TF32X3, 7),
                                       (swc.SWC_MODE_MIXED_TF32X3, 9),
                                       (swc.SWC_MODE_MIXED_BF16X3, 5),
                                       (swc.SWC_MODE_MIXED_BF16X3, 7),
                                       (swc.SWC_MODE_MIXED_BF16X3, 8)])
def test_split_plan_variants(cuda_ok, mode, plan):
    """The split factors under each of their execution-plan variants (0: right-looking
    tcgen05 updates scattered by FP64 atomics, trailing SYRK steps as tcgen05 tiles; 5: the
    trailing SYRK steps in FP64; 6, 7: tile-owner tcgen05 updates staged with TMA
    tile::gather4 loads or with cp.async; 8, 9: the right-looking products cut into tiles of
    256 or 128 columns of K) agree with the FP64 factor to FP32-class accuracy and refine to
    the FP64 backward error."""
    gs = load_sym("grid3d_24")
    A, _, _ = W.build("grid3d_24")
    P = W.assemble(A, gs["perm"], gs["super"])
    h = swc.Handle(0)
    h.set_plan(plan)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h.factor(P.A2x, swc.SWC_MODE_FP64) == 0
    L64 = h.get_L()
    assert h.factor(P.A2x, mode) == 0
    rel = np.abs(h.get_L() - L64).max() / np.abs(L64).max()
    assert 1e-12 < rel < 1e-5, rel
    b = np.random.default_rng(4).standard_normal(P.n)
    _, berr, _, _ = h.refine(b, tol=1e-14, maxit=30)
    assert berr.max() <= 1e-14
