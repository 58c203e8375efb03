"""Differentiable CBM products (no counterpart in the reference).

``cbm_apply(op, x)`` returns y = A_op x where A_op is the operator of a
cbm4mm / cbm4ad / cbm4dad instance; its backward computes A_op^T g in CBM
form: a reverse tree propagation (children summed into parents, deepest level
first) followed by a gather over the transposed delta matrix, both on the GPU
(cbm_matmul_adjoint).  Where the operator equals its transpose (a symmetric
A, as the undirected graphs of a GCN give, with A or D^-1/2 A D^-1/2), the
backward is the forward product itself: A^T g = A g, and the forward kernel
is the faster of the two.  No dense or torch.sparse matrix is formed.
"""
from __future__ import annotations

import torch

__all__ = ["cbm_apply", "CBMProduct"]

_PAIRS = {(torch.float32, torch.float32), (torch.bfloat16, torch.float32), (torch.bfloat16, torch.bfloat16)}


class CBMProduct(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, operator, out_dtype):
        x = x.contiguous()
        if (x.dtype, out_dtype) not in _PAIRS:
            raise RuntimeError(f"unsupported dtype pair {x.dtype} -> {out_dtype}")
        y = torch.empty(operator.plan.n_rows, x.shape[1], dtype=out_dtype, device=x.device)
        operator.matmul(x, y)
        ctx.operator = operator
        ctx.x_dtype = x.dtype
        return y

    @staticmethod
    def backward(ctx, g):
        op = ctx.operator
        g = g.contiguous()
        gdt = g.dtype if g.dtype in (torch.float32, torch.bfloat16) else torch.float32
        g = g.to(gdt)
        want = ctx.x_dtype
        ddt = want if (gdt, want) in _PAIRS else torch.float32
        dx = torch.empty(op.plan.n_cols, g.shape[1], dtype=ddt, device=g.device)
        if getattr(op, "self_adjoint", False):
            op.matmul(g, dx)
        else:
            op.adjoint(g, dx)
        return dx.to(want), None, None


def cbm_apply(operator, x, out_dtype=None):
    return CBMProduct.apply(x, operator, out_dtype or x.dtype)
