"""Differentiable projectors and an unrolled SQS-TV network (torch).

The forward projector and its exact transpose are each other's backward:

    y = A x      ->  dL/dx = A^T dL/dy
    x = A^T y    ->  dL/dy = A dL/dx

for the distance-driven fan/parallel pair (the back projector in exact-adjoint
mode) and the Siddon cone pair.  This is the role of the reference's
TensorFlow ops with their registered gradients
(projector/tensorflow/circular_2d.py:140-191, cone.py:193-236), rebuilt for
torch on the sm_100a kernels.

``UnrolledSQSTV`` unrolls SQS-TV iterations (ct_projector.recon
sqs_one_step with the TV prior) with a learnable step per iteration; each
iteration can be checkpointed (recomputed in backward) to bound memory.
"""
from __future__ import annotations

from typing import Optional, Sequence

import torch
from torch.utils.checkpoint import checkpoint

from . import _lib
from .projector import _device as D


# --------------------------------------------------------------------------- DD fan / parallel
class _DDFP(torch.autograd.Function):
    @staticmethod
    def forward(ctx, img, angles, projector, geom):
        ctx.projector, ctx.geom = projector, geom
        ctx.save_for_backward(angles)
        return D.dd_fp(projector, img, angles, geom)

    @staticmethod
    def backward(ctx, grad):
        (angles,) = ctx.saved_tensors
        g = D.dd_bp(ctx.projector, grad.contiguous(), angles, ctx.geom, adjoint=True) if ctx.needs_input_grad[0] else None
        return g, None, None, None


class _DDBP(torch.autograd.Function):
    @staticmethod
    def forward(ctx, prj, angles, projector, geom):
        ctx.projector, ctx.geom = projector, geom
        ctx.save_for_backward(angles)
        return D.dd_bp(projector, prj, angles, geom, adjoint=True)

    @staticmethod
    def backward(ctx, grad):
        (angles,) = ctx.saved_tensors
        g = D.dd_fp(ctx.projector, grad.contiguous(), angles, ctx.geom) if ctx.needs_input_grad[0] else None
        return g, None, None, None


def dd_fp(projector, img, angles, geom: str = "fan"):
    """Differentiable DD forward projection (geom 'fan' or 'parallel')."""
    return _DDFP.apply(img, angles, projector, _lib.GEOM_FAN if geom == "fan" else _lib.GEOM_PARALLEL)


def dd_bp(projector, prj, angles, geom: str = "fan"):
    """Differentiable exact transpose of dd_fp."""
    return _DDBP.apply(prj, angles, projector, _lib.GEOM_FAN if geom == "fan" else _lib.GEOM_PARALLEL)


# --------------------------------------------------------------------------- Siddon cone
class _SiddonFP(torch.autograd.Function):
    @staticmethod
    def forward(ctx, img, det_center, det_u, det_v, src, projector):
        ctx.projector = projector
        ctx.save_for_backward(det_center, det_u, det_v, src)
        return D.siddon_fp(projector, img, det_center, det_u, det_v, src)

    @staticmethod
    def backward(ctx, grad):
        geo = ctx.saved_tensors
        g = D.siddon_bp(ctx.projector, grad.contiguous(), *geo) if ctx.needs_input_grad[0] else None
        return g, None, None, None, None, None


class _SiddonBP(torch.autograd.Function):
    @staticmethod
    def forward(ctx, prj, det_center, det_u, det_v, src, projector):
        ctx.projector = projector
        ctx.save_for_backward(det_center, det_u, det_v, src)
        return D.siddon_bp(projector, prj, det_center, det_u, det_v, src)

    @staticmethod
    def backward(ctx, grad):
        geo = ctx.saved_tensors
        g = D.siddon_fp(ctx.projector, grad.contiguous(), *geo) if ctx.needs_input_grad[0] else None
        return g, None, None, None, None, None


def siddon_fp(projector, img, det_center, det_u, det_v, src):
    """Differentiable Siddon cone forward projection."""
    return _SiddonFP.apply(img, det_center, det_u, det_v, src, projector)


def siddon_bp(projector, prj, det_center, det_u, det_v, src):
    """Differentiable Siddon cone back projection (transpose of siddon_fp)."""
    return _SiddonBP.apply(prj, det_center, det_u, det_v, src, projector)


# --------------------------------------------------------------------------- TV prior (differentiable)
def tv_sqs_torch(img: torch.Tensor, weights: Sequence[float], eps: float = 1e-8):
    """(s1, s2, var) of the TV-SQS prior in torch ops, so gradients flow through
    it; same formula as the fused kernel (kernel/prior/cuda/TotalVariation.cu
    :21-149 of the reference)."""
    wz, wy, wx = (float(w) for w in weights)
    def bdiff(a, dim):
        n = a.shape[dim]
        first = torch.zeros_like(a.narrow(dim, 0, 1))
        return torch.cat([first, a.narrow(dim, 1, n - 1) - a.narrow(dim, 0, n - 1)], dim)

    def fdiff(a, dim):
        n = a.shape[dim]
        last = torch.zeros_like(a.narrow(dim, 0, 1))
        return torch.cat([a.narrow(dim, 0, n - 1) - a.narrow(dim, 1, n - 1), last], dim)

    def fshift(a, dim):  # value at index+1, the same value at the high border
        n = a.shape[dim]
        return torch.cat([a.narrow(dim, 1, n - 1), a.narrow(dim, n - 1, 1)], dim)

    dx, dy, dz = bdiff(img, 3), bdiff(img, 2), bdiff(img, 1)
    var = torch.sqrt(wx * dx * dx + wy * dy * dy + wz * dz * dz + eps)
    dx1, dy1, dz1 = fdiff(img, 3), fdiff(img, 2), fdiff(img, 1)
    varx, vary, varz = fshift(var, 3), fshift(var, 2), fshift(var, 1)
    s1 = (wx * dx + wy * dy + wz * dz) / var + wx * dx1 / varx + wy * dy1 / vary + wz * dz1 / varz
    s2 = (wx + wy + wz) / var + wx / varx + wy / vary + wz / varz
    return s1, s2, var


# --------------------------------------------------------------------------- unrolled SQS-TV
class UnrolledSQSTV(torch.nn.Module):
    """x_{k+1} = x_k - step_k (A^T (A x_k - y) + beta s1(x_k)) / (norm_img + beta s2(x_k))

    ``fp(x)`` / ``bp(y)`` are differentiable projector callables (for example
    ``lambda x: dd_fp(p, x, angles)``); ``norm_img`` = A^T A 1.  One learnable
    step per iteration (initialised to 1, the SQS step).  With ``checkpoint``
    each iteration's activations are recomputed during backward instead of
    stored."""

    def __init__(self, fp, bp, norm_img: torch.Tensor, n_iter: int = 4, beta: float = 1e-4,
                 tv_weights: Sequence[float] = (1.0, 1.0, 1.0), use_checkpoint: bool = True,
                 steps: Optional[Sequence[float]] = None):
        super().__init__()
        self.fp, self.bp = fp, bp
        self.register_buffer("norm_img", norm_img)
        self.beta = float(beta)
        self.tv_weights = tuple(tv_weights)
        self.use_checkpoint = use_checkpoint
        init = torch.ones(n_iter) if steps is None else torch.tensor(list(steps), dtype=torch.float32)
        self.steps = torch.nn.Parameter(init)

    def iteration(self, x, y, step):
        grad = self.bp(self.fp(x) - y)
        s1, s2, _ = tv_sqs_torch(x, self.tv_weights)
        return x - step * (grad + self.beta * s1) / (self.norm_img + self.beta * s2)

    def forward(self, x0: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
        x = x0
        for k in range(self.steps.numel()):
            if self.use_checkpoint and torch.is_grad_enabled():
                x = checkpoint(self.iteration, x, y, self.steps[k], use_reentrant=False)
            else:
                x = self.iteration(x, y, self.steps[k])
        return x
