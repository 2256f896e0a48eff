"""Equiangular fan-beam geometry, device arrays.

Same calls as ct_projector/projector/cupy/fan_equiangular.py of the reference:
ramp_filter (:19), fbp_bp (:74), distance_driven_fp (:129),
distance_driven_bp (:192).  Keyword-only extras: ``adjoint`` (exact transpose
of distance_driven_fp), ``out``, ``accumulate``, ``stream`` and ``dtype``
(bfloat16/float16 storage with FP32 accumulation).
"""
from __future__ import annotations

from typing import Union

from ... import _lib
from .. import _device as D
from .ct_projector import ct_projector


def ramp_filter(projector: ct_projector, prj, filter_type: str = "hann", *, exact: bool = False, out=None,
                stream=None):
    """Filter the projection for equiangular geometry; 'hamming', 'hann', 'cosine', else RL."""
    return D.like_input(D.ramp_filter(projector, prj, filter_type, _lib.GEOM_FAN, out=out, stream=stream,
                                      exact=exact), prj)


def fbp_bp(projector: ct_projector, prj, angles, *, out=None, accumulate=False, stream=None):
    """Pixel-driven fan back projection with the FBP distance weight.

    (The reference cupy wrapper binds the host-copy entry here with device
    pointers, fan_equiangular.py:95-97; this calls the device entry.)"""
    return D.like_input(D.fbp_bp(projector, prj, angles, out=out, accumulate=accumulate, stream=stream), prj)


def distance_driven_fp(projector: ct_projector, img, angles, branchless: Union[bool, int] = False, *, out=None,
                       stream=None, dtype=None):
    """Fan-beam forward projection, distance driven.  Returns [batch, nview, nv, nu]."""
    return D.like_input(D.dd_fp(projector, img, angles, _lib.GEOM_FAN, branchless, out=out, stream=stream,
                                dtype=dtype), img)


def distance_driven_bp(projector: ct_projector, prj, angles, is_fbp: Union[bool, int] = False,
                       branchless: Union[bool, int] = False, *, adjoint: bool = False, out=None, accumulate=False,
                       stream=None, dtype=None):
    """Fan-beam back projection, distance driven.  Returns [batch, nz, ny, nx].

    Default: the reference's normalised back projection; is_fbp selects the
    FBP weighting; adjoint=True gives the exact transpose of distance_driven_fp."""
    return D.like_input(D.dd_bp(projector, prj, angles, _lib.GEOM_FAN, is_fbp, branchless, adjoint, out=out,
                                accumulate=accumulate, stream=stream, dtype=dtype), prj)


def siddon_fp(projector: ct_projector, img, angles, *, out=None, stream=None):
    """Fan-beam forward projection, Siddon ray driven, on device arrays (the
    reference has it in its numpy module only, fan_equiangluar.py:131)."""
    return D.like_input(D.siddon_fan_fp(projector, img, angles, out=out, stream=stream), img)


def siddon_bp(projector: ct_projector, prj, angles, *, out=None, accumulate=False, stream=None):
    """Transpose of siddon_fp (reference numpy fan_equiangluar.py:185)."""
    return D.like_input(D.siddon_fan_bp(projector, prj, angles, out=out, accumulate=accumulate, stream=stream), prj)

