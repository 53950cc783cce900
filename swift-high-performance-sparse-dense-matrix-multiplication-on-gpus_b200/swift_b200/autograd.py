"""torch.autograd over the Swift products: Y = A(values) @ X with gradients for X and for the
nonzero values of A.

    plan = Plan.from_csr(rowptr, colidx, values, (M, K))
    Y = swift_spmm(plan, values, X)       # values: (nnz,) tensor, may require grad
    Y.sum().backward()                     # dX = A^T dY, dvalues[e] = dY[row_e] . X[col_e]

Forward runs swift_spmm; backward runs swift_spmm_transposed (dX) and swift_sddmm (dvalues),
each only when that input needs a gradient.  The plan's values follow `values`: every
forward loads them with swift_plan_set_values (a pass over the nonzeros that refreshes every
value copy of the format; in-place updates made through `.data` leave no trace on the
tensor, so no cache is trusted), and the backward reloads them only if another forward on the
same plan loaded different ones in between.  There is no counterpart in the reference, which
has no backward pass.
"""
from __future__ import annotations

import itertools

import torch

from .plan import Plan

_loads = itertools.count(1)


def _load_values(plan: Plan, values: torch.Tensor) -> int:
    plan.set_values(values)
    plan._autograd_load = next(_loads)
    return plan._autograd_load


class SwiftSpMMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, plan: Plan, values: torch.Tensor, X: torch.Tensor):
        ctx.load = _load_values(plan, values)
        Xc = X.contiguous()
        Y = plan.spmm(Xc)
        ctx.plan = plan
        ctx.save_for_backward(values, Xc)
        return Y

    @staticmethod
    def backward(ctx, dY):
        plan = ctx.plan
        values, X = ctx.saved_tensors
        dY = dY.contiguous().to(X.dtype)
        if getattr(plan, "_autograd_load", None) != ctx.load and ctx.needs_input_grad[2]:
            _load_values(plan, values)
        dvals = dX = None
        if ctx.needs_input_grad[2]:
            dX = plan.spmm_t(dY)
        if ctx.needs_input_grad[1]:
            dvals = plan.sddmm(dY, X).to(values.dtype)
        return None, dvals, dX


def swift_spmm(plan: Plan, values: torch.Tensor, X: torch.Tensor) -> torch.Tensor:
    """Y = A @ X where A has the plan's pattern and the given values (differentiable in both)."""
    return SwiftSpMMFunction.apply(plan, values, X)


class SwiftSparseLinear(torch.nn.Module):
    """Y = A @ X for a fixed sparsity pattern with trainable nonzero values (graph
    convolution, pruned layers)."""

    def __init__(self, rowptr, colidx, values, shape):
        super().__init__()
        v = torch.as_tensor(values)
        self.values = torch.nn.Parameter(v.detach().clone().cuda())
        self.plan = Plan.from_csr(rowptr, colidx, v.detach().cpu().numpy(), shape, build_transpose=True)

    def forward(self, X):
        return swift_spmm(self.plan, self.values, X)
