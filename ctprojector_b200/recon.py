"""SQS reconstruction driver (ct_projector.recon.cupy.sqs_algorithms of the
reference), on torch CUDA tensors.

``sqs_one_step`` (reference sqs_algorithms.py:22-57) performs one separable
quadratic surrogate update with a pluggable prior; ``nesterov_acceleration``
(:132-179) wraps any such step with Nesterov momentum.  The projector calls go
through ``projector.fp`` / ``projector.bp`` (the plug-in of ct_projector).
"""
from __future__ import annotations

from typing import Any, Callable, Tuple, Union

import torch


def sqs_one_step(projector, img, prj, norm_img, projector_norm: float, beta: float,
                 prior_func: Callable[..., Tuple[Any, ...]], prior_kwargs: dict, acc_fac: float = 1,
                 fp_kwargs: dict = None, bp_kwargs: dict = None, weight=None, return_loss: bool = False):
    """img <- img - (A^T w (A img - prj) acc_fac + beta s1) / (norm_img + beta s2)."""
    fp_kwargs = fp_kwargs or {}
    bp_kwargs = bp_kwargs or {}
    if weight is None:
        weight = 1
    fp = projector.fp(img, **fp_kwargs) / projector_norm
    fp = fp - prj / projector_norm
    bp = projector.bp(fp * weight, **bp_kwargs) / projector_norm
    prior_kwargs["img"] = img
    prior_res = prior_func(**prior_kwargs)
    img = img - (bp * acc_fac + beta * prior_res[0]) / (norm_img + beta * prior_res[1])
    if return_loss:
        fp = projector.fp(img) / projector_norm
        data_loss = 0.5 * torch.sum(weight * (fp - prj / projector_norm) ** 2)
        prior_loss = torch.sum(prior_res[2])
        return img, data_loss, prior_loss
    return img


def nesterov_acceleration(recon_func: Callable[..., Union[Any, Tuple[Any, ...]]], recon_kwargs: dict, img,
                          img_nesterov, nesterov: float = 0.5):
    """One accelerated step: x* = f(img); img <- x* + nesterov (x* - img_nesterov)."""
    recon_kwargs["img"] = img
    res = recon_func(**recon_kwargs)
    if isinstance(res, tuple):
        img = res[0] + nesterov * (res[0] - img_nesterov)
        img_nesterov = res[0]
        return tuple([img, img_nesterov] + list(res[1:]))
    img = res + nesterov * (res - img_nesterov)
    return img, res


def sqs_tv_update(x: torch.Tensor, bp: torch.Tensor, norm: torch.Tensor, beta: float,
                  weights=(1.0, 1.0, 1.0), eps: float = 1e-8, zlink: torch.Tensor = None, out: torch.Tensor = None,
                  x_lp: torch.Tensor = None, stream=None) -> torch.Tensor:
    """One fused SQS-TV iteration on a flat slice array x [nslices, ny, nx]
    (any leading shape whose product is the slice count):

        out = x - (bp + beta s1(x)) / (norm + beta s2(x))

    with the TV-SQS terms of ``prior.tv_sqs`` (weights along z, y, x).  ``zlink``
    (uint8 per slice, bit 0 / bit 1 = z neighbour below / above in the same
    volume; None = no z coupling) lets volumes of different depths share one
    array.  ``norm`` holds k slices read at slice i % k (one slice broadcasts).
    ``x_lp`` (bf16 or fp16, same shape) also receives the result."""
    from ctypes import c_float, c_size_t, c_uint, c_void_p

    from . import _lib
    from .projector._device import ptr, stream_handle

    nx, ny = int(x.shape[-1]), int(x.shape[-2])
    ns = x.numel() // (nx * ny)
    for name, t in (("x", x), ("bp", bp), ("norm", norm)):
        if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
    if bp.numel() != x.numel() or norm.numel() % (nx * ny):
        raise ValueError("bp must match x and norm must hold whole slices")
    out = torch.empty_like(x) if out is None else out
    flags = 0
    if x_lp is not None:
        flags = {torch.bfloat16: _lib.FLAG_OUT_BF16, torch.float16: _lib.FLAG_OUT_FP16}[x_lp.dtype]
    if zlink is not None and (zlink.dtype != torch.uint8 or zlink.numel() != ns):
        raise ValueError("zlink must be uint8 with one entry per slice")
    wz, wy, wx = (float(w) for w in weights)
    _lib.check(_lib.lib().ctp_sqs_tv_update(
        ptr(out), ptr(x_lp) if x_lp is not None else c_void_p(0), ptr(x), ptr(bp), ptr(norm),
        c_size_t(norm.numel() // (nx * ny)), ptr(zlink) if zlink is not None else c_void_p(0), c_float(wx),
        c_float(wy), c_float(wz), c_float(beta), c_float(eps), c_size_t(nx), c_size_t(ny), c_size_t(ns),
        c_uint(flags), stream_handle(stream, x.device)), "sqs_tv_update")
    return out
