"""torch.autograd wrappers over the library's adjoint (a thin test shim).

``LogDet.apply(values, handle, mode)`` returns log det A for the stored nonzeros ``values``
(a CUDA float64 tensor in the analysed structure of ``handle``); its backward is
``swc_logdet_grad``.  ``Solve.apply(values, b, handle, mode, tol)`` returns x = A^{-1} b
(refined to backward error ``tol``); its backward solves lam = A^{-1} grad_x and returns
(``swc_solve_grad``(x, lam), lam).  Both factor in forward; the handle keeps that factor
for backward, so a handle serves one forward/backward pair at a time.
"""
from __future__ import annotations

import torch

from . import SWC_MODE_FP64, SWCError


class LogDet(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, handle, mode=SWC_MODE_FP64):
        info = handle.factor(values, mode)
        if info:
            raise SWCError(1, f"matrix is not positive definite (column {info - 1})")
        ctx.handle = handle
        return torch.tensor(handle.logdet(), dtype=torch.float64, device=values.device)

    @staticmethod
    def backward(ctx, g):
        h = ctx.handle
        grad = torch.empty(h.nnz, dtype=torch.float64, device=g.device)
        h.logdet_grad(grad)
        return g * grad, None, None


class Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, b, handle, mode=SWC_MODE_FP64, tol=1e-15):
        info = handle.factor(values, mode)
        if info:
            raise SWCError(1, f"matrix is not positive definite (column {info - 1})")
        x, _, _, _ = handle.refine(b.contiguous(), tol=tol, maxit=30)
        ctx.handle = handle
        ctx.tol = tol
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, gx):
        (x,) = ctx.saved_tensors
        h = ctx.handle
        lam, _, _, _ = h.refine(gx.contiguous(), tol=ctx.tol, maxit=30)
        grad = h.solve_grad(x, lam)
        return grad, lam, None, None, None
