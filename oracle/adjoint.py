"""TEST ORACLE ONLY -- dense FP64 gradients for checking the library's adjoint.

For A SPD with its lower triangle stored (symmetric storage: a stored off-diagonal value
a_p at (i, j), i > j, stands for both A_ij and A_ji):

* d log det A / d a_p = (A^{-1})_ij (2 - delta_ij)   (d log det A = tr(A^{-1} dA));
* for f(x), x = A^{-1} b, with lam = A^{-1} df/dx:
  d f / d a_p = -(lam_i x_j + lam_j x_i), or -lam_i x_i on the diagonal.

Plain numpy on a dense copy of A (n up to a few thousand).  Only tests import this module.
"""
from __future__ import annotations

import numpy as np


def dense_from_lower(n, Ap, Ai, Ax):
    A = np.zeros((n, n))
    for j in range(n):
        for p in range(Ap[j], Ap[j + 1]):
            i = Ai[p]
            A[i, j] = Ax[p]
            A[j, i] = Ax[p]
    return A


def pattern_ij(n, Ap, Ai):
    cols = np.repeat(np.arange(n), np.diff(np.asarray(Ap)))
    return np.asarray(Ai), cols


def logdet_grad(n, Ap, Ai, Ax):
    A = dense_from_lower(n, Ap, Ai, Ax)
    Z = np.linalg.inv(A)
    i, j = pattern_ij(n, Ap, Ai)
    return Z[i, j] * np.where(i == j, 1.0, 2.0)


def solve_loss_grad(n, Ap, Ai, Ax, b, y):
    """f = 0.5 ||A^{-1} b - y||^2: returns (f, df/dvalues, df/db)."""
    A = dense_from_lower(n, Ap, Ai, Ax)
    x = np.linalg.solve(A, b)
    lam = np.linalg.solve(A, x - y)
    i, j = pattern_ij(n, Ap, Ai)
    g = np.where(i == j, -lam[i] * x[j], -(lam[i] * x[j] + lam[j] * x[i]))
    return 0.5 * float(np.dot(x - y, x - y)), g, lam
