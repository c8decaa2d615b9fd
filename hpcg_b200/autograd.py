"""A thin torch.autograd.Function over the solve, for checking the implicit
adjoint (hpcg_b200_adjoint) against finite differences and a host adjoint.

    x = HpcgSolve.apply(values27, b, problem, tol, max_iter)

values27: float64 [n, 27] fine-level values in the layout of
hpcg_b200_set_values (natural rows, direction slots); b: float64 [n]. The
forward pass loads the values into the problem's fine level and runs the
preconditioned CG from x = 0 to `tol`; the backward pass runs the adjoint solve
with the same hierarchy and returns (dL/dvalues27, dL/db). Only x is saved for
the backward pass.
"""
from __future__ import annotations

import torch


class HpcgSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values27, b, problem, tol=1e-10, max_iter=1000):
        problem.set_values(0, values27.detach().contiguous())
        x = torch.zeros_like(b)
        problem.CG(b.detach().contiguous(), x, max_iter, tol, True)
        ctx.save_for_backward(x)
        ctx.problem, ctx.tol, ctx.max_iter = problem, tol, max_iter
        ctx.shape = values27.shape
        return x

    @staticmethod
    def backward(ctx, grad_x):
        (x,) = ctx.saved_tensors
        grad_b = torch.empty_like(x)
        grad_v = torch.empty(ctx.shape, dtype=torch.float64, device=x.device)
        ctx.problem.adjoint(x, grad_x.contiguous(), ctx.max_iter, ctx.tol, grad_b, grad_v)
        return grad_v, grad_b, None, None, None
