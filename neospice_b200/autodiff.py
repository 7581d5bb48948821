"""Differentiable batched DC operating point and transient loss.

``dc_solve(batch, params)`` returns the packed solutions of every instance of
a ``DcBatch`` for the packed parameter tensor ``params`` and is a
``torch.autograd.Function``: its backward runs the batched adjoint (the
Jacobian at the solution, the transposed solve on its factors and the
parameter contraction, all on the GPU) and returns dL/dparams for
resistances, DC source values and MOSFET W, L and VTO (zero for the other
entries of the parameter blocks).

``tran_loss(batch, probes, targets, params)`` returns, per instance of a
recorded ``TranBatch``, L_i = weight * sum_n (x_n[probe_i] - target_n)^2 over
the recorded timepoints, and its backward is the transient adjoint (a
transposed solve on each step's LU, checkpointed replay, capacitor, diode
and level-1 MOSFET charge recursion) with respect to resistances,
capacitances, DC source values and MOSFET W, L and VTO.

Failed instances do not produce silent garbage: an instance whose forward
solve did not converge (status != 0) gets NaN solutions / loss, and an
instance whose forward or adjoint status is not 0 gets NaN gradients in its
own parameter slice; the other instances are unaffected.
"""
from __future__ import annotations

import numpy as np
import torch


def _nan_slices(t, offsets, bad):
    """Set t[offsets[i]:offsets[i+1]] = NaN for every instance i in bad."""
    for i in bad:
        t[int(offsets[i]):int(offsets[i + 1])] = float("nan")


def _failed(status):
    return np.nonzero(status.cpu().numpy() != 0)[0].tolist()


class _DcSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, batch):
        p = params.detach().contiguous()
        sols, status, _ = batch.run(d_params=p)
        bad = _failed(status)
        _nan_slices(sols, batch.solution_offsets, bad)
        ctx.batch = batch
        ctx.bad = bad
        ctx.save_for_backward(p, sols)
        return sols

    @staticmethod
    def backward(ctx, grad_sols):
        p, sols = ctx.saved_tensors
        batch = ctx.batch
        grads, status = batch.adjoint(sols, grad_sols.contiguous(), d_params=p)
        bad = sorted(set(ctx.bad) | set(_failed(status)))
        _nan_slices(grads, batch.param_offsets, bad)
        return grads, None


def dc_solve(batch, params: torch.Tensor) -> torch.Tensor:
    """Packed DC solutions of ``batch`` at ``params`` (differentiable)."""
    return _DcSolve.apply(params, batch)


class _TranLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, batch, probes, targets, weight, every):
        off, p_dc, p_tr = batch.params()
        d_dc = params.detach().contiguous()
        # The transient's parameter vector differs from the DC one only where
        # PULSE defaults are resolved (source timing, never differentiated):
        # take those entries from the batch, the rest from params.
        resolved = torch.from_numpy(p_dc != p_tr).cuda()
        d_tr = torch.where(resolved, torch.from_numpy(p_tr).cuda(), d_dc)
        grads, loss, status = batch.adjoint(probes, targets, weight, every, d_dc, d_tr)
        bad = _failed(status)
        _nan_slices(grads, off, bad)
        for i in bad:
            loss[i] = float("nan")
        ctx.offsets = off
        ctx.save_for_backward(grads)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):
        (grads,) = ctx.saved_tensors
        off = torch.from_numpy(np.diff(ctx.offsets)).to(grads.device)
        scale = torch.repeat_interleave(grad_loss.to(grads.dtype), off)
        return grads * scale, None, None, None, None, None


def tran_loss(batch, probes, targets: torch.Tensor, params: torch.Tensor | None = None,
              weight: float = 1.0, every: int = 32) -> torch.Tensor:
    """Per-instance loss weight * sum_n (x_n[probes[i]] - targets_n)^2 of a
    recorded ``TranBatch`` (``batch.record(True); batch.run()`` first),
    replayed at ``params`` (packed like ``batch.params()``'s DC vector; None:
    the batch's own, and no gradient flows).  ``targets`` holds
    ``max_points`` values per instance, at the recorded timepoints.
    Differentiable with respect to ``params`` (R, C, DC sources, MOSFET W / L /
    VTO)."""
    probes = np.ascontiguousarray(probes, np.int32)
    if params is None:
        _, p_dc, _ = batch.params()
        with torch.no_grad():
            return _TranLoss.forward(_Ctx(), torch.from_numpy(p_dc).cuda(), batch, probes,
                                     targets.contiguous(), float(weight), int(every))
    return _TranLoss.apply(params, batch, probes, targets.contiguous(), float(weight), int(every))


class _Ctx:
    """Stand-in autograd context for a forward evaluated without a graph."""

    def save_for_backward(self, *tensors):
        self.saved_tensors = tensors
