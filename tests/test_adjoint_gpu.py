"""Adjoint on the GPU: gradients of log det A and of 0.5 ||A^{-1} b - y||^2 with respect to
the stored nonzeros of A, against the dense FP64 oracle (40 x 40 GMRF) and against central
finite differences of the library's own factorization (500 x 500 GMRF)."""
import numpy as np
import pytest

from conftest import load_sym

pytestmark = pytest.mark.gpu


def gmrf_problem(k):
    from swcholesky_b200 import workloads as W
    A, perm, _ = W.build(f"gmrf_{k}")
    return W.assemble_own(A, perm)


def handle_for(P):
    import swcholesky_b200 as S
    h = S.Handle(0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    return h


@pytest.fixture(scope="module")
def gmrf40():
    return gmrf_problem(40)


def test_logdet_and_grad_dense(cuda_ok, gmrf40):
    from oracle import adjoint as OA
    P = gmrf40
    h = handle_for(P)
    assert h.factor(P.A2x) == 0
    ref = np.linalg.slogdet(OA.dense_from_lower(P.n, P.A2p, P.A2i, P.A2x))[1]
    assert abs(h.logdet() - ref) <= 1e-12 * abs(ref)
    g = h.logdet_grad()
    gr = OA.logdet_grad(P.n, P.A2p, P.A2i, P.A2x)
    assert np.max(np.abs(g - gr)) <= 1e-10 * np.max(np.abs(gr))
    # twice in a row: identical (deterministic sweep)
    np.testing.assert_array_equal(h.logdet_grad(), g)


def test_solve_grad_dense(cuda_ok, gmrf40):
    from oracle import adjoint as OA
    P = gmrf40
    h = handle_for(P)
    assert h.factor(P.A2x) == 0
    rng = np.random.default_rng(7)
    b, y = rng.standard_normal(P.n), rng.standard_normal(P.n)
    _, gr, lam_r = OA.solve_loss_grad(P.n, P.A2p, P.A2i, P.A2x, b, y)
    x, _, _, _ = h.refine(b, tol=1e-15)
    lam, _, _, _ = h.refine(x - y, tol=1e-15)
    assert np.max(np.abs(lam - lam_r)) <= 1e-10 * np.max(np.abs(lam_r))
    g = h.solve_grad(x, lam)
    assert np.max(np.abs(g - gr)) <= 1e-10 * np.max(np.abs(gr))


def test_mixed_factor_grad_dense(cuda_ok, gmrf40):
    """Split-TF32 Schur updates: log det gradient within 1e-4 of the dense FP64 one (FP32-class
    factor); the solve gradient, through FP64 refinement, within 1e-10."""
    import swcholesky_b200 as S
    from oracle import adjoint as OA
    P = gmrf40
    h = handle_for(P)
    assert h.factor(P.A2x, S.SWC_MODE_MIXED_TF32X3) == 0
    gr = OA.logdet_grad(P.n, P.A2p, P.A2i, P.A2x)
    err = np.max(np.abs(h.logdet_grad() - gr)) / np.max(np.abs(gr))
    assert err <= 1e-4, err
    rng = np.random.default_rng(7)
    b, y = rng.standard_normal(P.n), rng.standard_normal(P.n)
    _, gs, _ = OA.solve_loss_grad(P.n, P.A2p, P.A2i, P.A2x, b, y)
    x, _, _, _ = h.refine(b, tol=1e-15)
    lam, _, _, _ = h.refine(x - y, tol=1e-15)
    assert np.max(np.abs(h.solve_grad(x, lam) - gs)) <= 1e-10 * np.max(np.abs(gs))


def test_autograd_shim(cuda_ok, gmrf40):
    import torch
    from oracle import adjoint as OA
    from swcholesky_b200.autograd import LogDet, Solve
    P = gmrf40
    h = handle_for(P)
    v = torch.tensor(P.A2x, dtype=torch.float64, device="cuda", requires_grad=True)
    LogDet.apply(v, h).backward()
    gr = OA.logdet_grad(P.n, P.A2p, P.A2i, P.A2x)
    assert np.max(np.abs(v.grad.cpu().numpy() - gr)) <= 1e-10 * np.max(np.abs(gr))
    rng = np.random.default_rng(11)
    b, y = rng.standard_normal(P.n), rng.standard_normal(P.n)
    _, gs, lam_r = OA.solve_loss_grad(P.n, P.A2p, P.A2i, P.A2x, b, y)
    v.grad = None
    bt = torch.tensor(b, dtype=torch.float64, device="cuda", requires_grad=True)
    yt = torch.tensor(y, dtype=torch.float64, device="cuda")
    x = Solve.apply(v, bt, h)
    (0.5 * ((x - yt) ** 2).sum()).backward()
    assert np.max(np.abs(v.grad.cpu().numpy() - gs)) <= 1e-10 * np.max(np.abs(gs))
    assert np.max(np.abs(bt.grad.cpu().numpy() - lam_r)) <= 1e-10 * np.max(np.abs(lam_r))


def _fd4(f, h):
    """Fourth-order central difference (-f(2h) + 8 f(h) - 8 f(-h) + f(-2h)) / 12h."""
    return (-f(2 * h) + 8 * f(h) - 8 * f(-h) + f(-2 * h)) / (12 * h)


@pytest.fixture(scope="module")
def gmrf500():
    from swcholesky_b200 import workloads as W
    g = load_sym("gmrf_500")
    A, _, _ = W.build("gmrf_500")
    return W.assemble(A, g["perm"], g["super"])


def _rel(fd, ad):
    """|fd - ad| / |ad| per sample (plain relative error; a sample with ad = 0 counts its
    absolute error)."""
    fd, ad = np.asarray(fd), np.asarray(ad)
    den = np.abs(ad)
    return np.abs(fd - ad) / np.where(den > 0, den, 1.0)


def test_fd_logdet_gmrf500(cuda_ok, gmrf500):
    import torch
    P = gmrf500
    h = handle_for(P)
    v = torch.tensor(P.A2x, dtype=torch.float64, device="cuda")
    assert h.factor(v) == 0
    g = h.logdet_grad()
    rng = np.random.default_rng(2024)
    idx = rng.choice(P.A2x.size, 64, replace=False)
    fds = []
    for p in idx:
        a = float(P.A2x[p])

        def f(d):
            v[p] = a + d
            assert h.factor(v) == 0
            return h.logdet()

        fds.append(_fd4(f, 1e-3 * max(abs(a), 1.0)))
        v[p] = a
    rel = _rel(fds, g[idx])
    assert rel.max() <= 1e-6, rel.max()


@pytest.mark.parametrize("mode", [0, 1])
def test_fd_solve_loss_gmrf500(cuda_ok, gmrf500, mode):
    """mode 1: split-TF32 Schur updates, FP64 diagonal blocks and FP64 refinement."""
    import torch
    P = gmrf500
    h = handle_for(P)
    rng = np.random.default_rng(99)
    b = torch.tensor(rng.standard_normal(P.n), dtype=torch.float64, device="cuda")
    y = torch.tensor(rng.standard_normal(P.n), dtype=torch.float64, device="cuda")
    v = torch.tensor(P.A2x, dtype=torch.float64, device="cuda")

    def loss():
        assert h.factor(v, mode) == 0
        x, berr, _, _ = h.refine(b, tol=1e-16, maxit=30)
        return x, 0.5 * float(torch.dot(x - y, x - y))

    x, _ = loss()
    lam, _, _, _ = h.refine((x - y).contiguous(), tol=1e-16, maxit=30)
    g = h.solve_grad(x, lam).cpu().numpy()
    idx = rng.choice(P.A2x.size, 64, replace=False)
    fds = []
    for p in idx:
        a = float(P.A2x[p])

        def f(d):
            v[p] = a + d
            return loss()[1]

        fds.append(_fd4(f, 1e-3 * max(abs(a), 1.0)))
        v[p] = a
    rel = _rel(fds, g[idx])
    assert rel.max() <= 1e-6, rel.max()
