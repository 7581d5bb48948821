"""Differentiable batched DC operating point.

``dc_solve(batch, params)`` returns the packed solutions of every instance of
a ``DcBatch`` for the packed parameter tensor ``params`` and is a
``torch.autograd.Function``: its backward runs the batched adjoint (the
Jacobian at the solution, the transposed solve on its factors and the
parameter contraction, all on the GPU) and returns dL/dparams for
resistances, DC source values and MOSFET W, L and VTO (zero for the other
entries of the parameter blocks).
"""
from __future__ import annotations

import torch


class _DcSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, batch):
        p = params.detach().contiguous()
        sols, status, _ = batch.run(d_params=p)
        ctx.batch = batch
        ctx.status = status
        ctx.save_for_backward(p, sols)
        return sols

    @staticmethod
    def backward(ctx, grad_sols):
        p, sols = ctx.saved_tensors
        grads, status = ctx.batch.adjoint(sols, grad_sols.contiguous(), d_params=p)
        return grads, None


def dc_solve(batch, params: torch.Tensor) -> torch.Tensor:
    """Packed DC solutions of ``batch`` at ``params`` (differentiable)."""
    return _DcSolve.apply(params, batch)
