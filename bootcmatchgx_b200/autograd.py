"""torch.autograd binding of the FCG + BCMG solve x = A^{-1} b.

The forward pass is bcmgx_solve; the backward pass is bcmgx_solve_adjoint, which reuses the
forward hierarchy to solve A lambda = dL/dx (A is SPD) and forms dL/db = lambda and
dL/dA_ij = -lambda_i x_j on A's sparsity pattern, all in libbcmgx.so. Gradients flow to the CSR
value array and to b; the pattern (row, col) is not differentiable.
"""
from __future__ import annotations

import torch

from .api import Hierarchy, params_default


class SparseSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, val, b, hierarchy):
        x, info = hierarchy.solve(b.detach().contiguous())
        ctx.hierarchy = hierarchy
        ctx.info = info
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, gx):
        (x,) = ctx.saved_tensors
        need_a, need_b = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_a or need_b):
            return None, None, None
        lam, dA, _ = ctx.hierarchy.adjoint(gx.detach().contiguous(), x if need_a else None, want_dA=need_a)
        return (dA if need_a else None), (lam if need_b else None), None


def default_params(**kw):
    base = dict(solver="FCG", preconditioner="BCMG", rtol=1e-10, dispnorm=0)
    base.update(kw)
    return params_default(**base)


def solve(row, col, val, b, params=None, hierarchy=None):
    """x = A^{-1} b, differentiable with respect to val (the CSR values) and b.

    row, col, val, b are CUDA tensors (int32, int32, float64, float64). The hierarchy is built
    from val.detach() unless one built for the same values is passed in. The backward pass uses
    the hierarchy's FCG settings (rtol) for the adjoint solve.
    """
    if hierarchy is None:
        hierarchy = Hierarchy(row, col, val.detach(), params or default_params())
    return SparseSolve.apply(val, b, hierarchy)
