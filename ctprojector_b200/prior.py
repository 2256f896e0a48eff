"""Priors for SQS reconstruction (ct_projector.prior.cupy of the reference).

``tv_sqs`` returns the separable-quadratic-surrogate terms of the anisotropic
total-variation prior (reference prior/cupy/recon_prior.py:85-135 and
kernel/prior/cuda/TotalVariation.cu:21-149), computed by one fused sm_100a
kernel on the caller's stream.
"""
from __future__ import annotations

from ctypes import c_float, c_size_t
from typing import Tuple

import torch

from ._lib import check, lib
from .projector._device import as_tensor, like_input, ptr, stream_handle


def tv_sqs(img, weights: Tuple[float, float, float], eps: float = 1e-8, *, stream=None):
    """(s1, s2, var) for img [batch, nz, ny, nx]; weights along (z, y, x).

    s1 is the surrogate's first-order term, s2 its curvature, var the
    variation map sqrt(wx dx^2 + wy dy^2 + wz dz^2 + eps)."""
    t = as_tensor(img, lowp_ok=False)
    nb, nz, ny, nx = t.shape
    s1 = torch.empty_like(t)
    s2 = torch.empty_like(t)
    var = torch.empty_like(t)
    check(lib().ctp_tv_sqs(ptr(s1), ptr(s2), ptr(var), ptr(t), c_float(weights[2]), c_float(weights[1]),
                           c_float(weights[0]), c_size_t(nb), c_size_t(nx), c_size_t(ny), c_size_t(nz),
                           c_float(eps), stream_handle(stream, t.device)), "tv_sqs")
    return like_input(s1, img), like_input(s2, img), like_input(var, img)
