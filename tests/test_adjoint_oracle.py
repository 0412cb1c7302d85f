"""The dense adjoint oracle (oracle/adjoint.py) against central finite differences."""
import numpy as np

from oracle import adjoint as OA
from swcholesky_b200 import matrices as M


def small_gmrf(k=6, seed=3):
    A = M.weighted_grid_2d(k, sigma=0.7, shift=0.1, seed=seed)
    return A.n, A.indptr, A.indices, A.data.copy()


def test_logdet_grad_vs_fd():
    n, Ap, Ai, Ax = small_gmrf()
    g = OA.logdet_grad(n, Ap, Ai, Ax)
    rng = np.random.default_rng(0)
    for p in rng.choice(Ax.size, 12, replace=False):
        h = 1e-5
        vals = []
        for s in (+1, -1):
            X = Ax.copy()
            X[p] += s * h
            vals.append(np.linalg.slogdet(OA.dense_from_lower(n, Ap, Ai, X))[1])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[p]) <= 1e-7 * max(1.0, abs(g[p]))


def test_solve_loss_grad_vs_fd():
    n, Ap, Ai, Ax = small_gmrf()
    rng = np.random.default_rng(1)
    b, y = rng.standard_normal(n), rng.standard_normal(n)
    f0, g, lam = OA.solve_loss_grad(n, Ap, Ai, Ax, b, y)
    for p in rng.choice(Ax.size, 12, replace=False):
        h = 1e-5
        vals = []
        for s in (+1, -1):
            X = Ax.copy()
            X[p] += s * h
            vals.append(OA.solve_loss_grad(n, Ap, Ai, X, b, y)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g[p]) <= 1e-6 * max(1.0, abs(g[p]))
    # df/db = lam
    q = 5
    bb = b.copy()
    bb[q] += 1e-6
    f1 = OA.solve_loss_grad(n, Ap, Ai, Ax, bb, y)[0]
    bb[q] -= 2e-6
    f2 = OA.solve_loss_grad(n, Ap, Ai, Ax, bb, y)[0]
    assert abs((f1 - f2) / 2e-6 - lam[q]) <= 1e-6 * max(1.0, abs(lam[q]))
