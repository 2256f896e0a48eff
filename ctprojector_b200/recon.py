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
