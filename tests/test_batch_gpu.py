"""Batched factorization: independent matrices of uneven size as one block-diagonal
structure, factored by one graph replay (persistent small-supernode walk + level launches),
against per-matrix dense / sparse FP64 references."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_batch(count=12, seed=5):
    from swcholesky_b200 import workloads as W
    return W.batch_matrices(count=count, seed=seed, lo=5, hi=40)


def concat_values(mats):
    return np.concatenate([m.data for m in mats])


def per_matrix_solve(mats, b):
    import scipy.sparse.linalg as sla
    out, o = [], 0
    for m in mats:
        out.append(sla.spsolve(m.to_scipy_full().tocsc(), b[o:o + m.n]))
        o += m.n
    return np.concatenate(out)


def test_batch_fp64_solve_and_logdet(cuda_ok):
    import swcholesky_b200 as S
    mats, _ = small_batch()
    h = S.Handle(0)
    h.batch_analyze(mats)
    assert h.n == sum(m.n for m in mats)
    assert h.factor(concat_values(mats)) == 0
    rng = np.random.default_rng(1)
    b = rng.standard_normal(h.n)
    x = h.solve(b)
    xr = per_matrix_solve(mats, b)
    assert np.max(np.abs(x - xr)) <= 1e-10 * np.max(np.abs(xr))
    berr = h.batch_berr(b, x)
    assert berr.shape == (len(mats),) and berr.max() <= 1e-13
    ld = sum(np.linalg.slogdet(m.to_scipy_full().toarray())[1] for m in mats)
    assert abs(h.logdet() - ld) <= 1e-12 * abs(ld)


def test_batch_not_spd_reports_column(cuda_ok):
    import swcholesky_b200 as S
    mats, _ = small_batch(count=4)
    h = S.Handle(0)
    h.batch_analyze(mats)
    v = concat_values(mats)
    # make the third matrix indefinite at its first stored diagonal
    o = sum(int(m.indptr[-1]) for m in mats[:2])
    v[o] = -1.0
    info = h.factor(v)
    first = sum(m.n for m in mats[:2])
    assert info >= first + 1 and info <= first + mats[2].n


def test_batch_autotune_and_cache(cuda_ok, tmp_path):
    import swcholesky_b200 as S
    mats, _ = small_batch(count=24, seed=9)
    v = concat_values(mats)
    h = S.Handle(0)
    h.batch_analyze(mats)
    cache = str(tmp_path / "tune.txt")
    choice, ms = h.batch_autotune(v, S.SWC_MODE_FP64, cache)
    assert 0 <= choice[0] < 3 and 0 <= choice[1] < 5 and ms > 0   # plans 5-7: mixed modes
    # the tuned handle factors and solves correctly
    assert h.factor(v) == 0
    b = np.random.default_rng(3).standard_normal(h.n)
    x, berr, _, _ = h.refine(b, tol=1e-14)
    assert h.batch_berr(b, x).max() <= 1e-14
    # second run on a new handle reads the cache
    h2 = S.Handle(0)
    h2.batch_analyze(mats)
    choice2, ms2 = h2.batch_autotune(v, S.SWC_MODE_FP64, cache)
    assert choice2 == choice and ms2 == pytest.approx(ms, rel=1e-5)


def test_config_batch256_both_modes(cuda_ok):
    """256 grids with sides in [30, 200]: FP64 and split-TF32 factorizations, refined solve,
    per-matrix backward error <= 1e-12."""
    import torch
    import swcholesky_b200 as S
    from swcholesky_b200 import workloads as W
    mats, sides = W.batch_matrices()
    assert len(mats) == 256 and sides.min() >= 30 and sides.max() <= 200
    h = S.Handle(0)
    h.batch_analyze(mats)
    v = torch.tensor(concat_values(mats), dtype=torch.float64, device="cuda")
    b = torch.tensor(np.random.default_rng(0).standard_normal(h.n), dtype=torch.float64,
                     device="cuda")
    for mode in (S.SWC_MODE_FP64, S.SWC_MODE_MIXED_TF32X3):
        assert h.factor(v, mode) == 0
        x, berr, _, _ = h.refine(b, tol=1e-14, maxit=30)
        per = h.batch_berr(b, x)
        assert per.max() <= 1e-12, (mode, per.max())
