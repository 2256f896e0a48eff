"""Parallel-beam geometry, device arrays.

Same calls as ct_projector/projector/cupy/parallel.py of the reference:
ramp_filter (:19), distance_driven_fp (:73), distance_driven_bp (:132).
"""
from __future__ import annotations

from typing import Union

from ... import _lib
from .. import _device as D
from .ct_projector import ct_projector


def ramp_filter(projector: ct_projector, prj, filter_type: str = "hann", *, exact: bool = False, out=None,
                stream=None):
    """Filter the projection for parallel geometry; 'hamming', 'hann', 'cosine', else RL."""
    return D.like_input(D.ramp_filter(projector, prj, filter_type, _lib.GEOM_PARALLEL, out=out, stream=stream,
                                      exact=exact), prj)


def distance_driven_fp(projector: ct_projector, img, angles, branchless: Union[bool, int] = False, *, out=None,
                       stream=None, dtype=None):
    """Parallel-beam forward projection, distance driven.  Returns [batch, nview, nv, nu]."""
    return D.like_input(D.dd_fp(projector, img, angles, _lib.GEOM_PARALLEL, branchless, out=out, stream=stream,
                                dtype=dtype), img)


def distance_driven_bp(projector: ct_projector, prj, angles, is_fbp: Union[bool, int] = False,
                       branchless: Union[bool, int] = False, *, adjoint: bool = False, out=None, accumulate=False,
                       stream=None, dtype=None):
    """Parallel-beam back projection, distance driven.  Returns [batch, nz, ny, nx]."""
    return D.like_input(D.dd_bp(projector, prj, angles, _lib.GEOM_PARALLEL, is_fbp, branchless, adjoint, out=out,
                                accumulate=accumulate, stream=stream, dtype=dtype), prj)


def pixel_driven_bp(projector: ct_projector, prj, angles, *, out=None, accumulate=False, stream=None):
    """Pixel-driven parallel back projection on device arrays (the reference
    has it in its numpy module only, parallel.py:75)."""
    return D.like_input(D.pixel_bp_parallel(projector, prj, angles, out=out, accumulate=accumulate, stream=stream),
                        prj)

