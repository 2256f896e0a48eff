"""Tomosynthesis geometry (detector u = (1,0,0), v = (0,1,0)), device arrays.

Same calls as ct_projector/projector/cupy/tomo.py of the reference:
distance_driven_fp (:15), distance_driven_bp (:85), filter_fbp (:157).  ``branchless`` selects
the same operator (both are the exact box integral).
"""
from __future__ import annotations

from .. import _device as D
from .ct_projector import ct_projector


def distance_driven_fp(projector: ct_projector, img, det_center, src, branchless: bool = False, *, out=None,
                       stream=None):
    return D.like_input(D.tomo_fp(projector, img, det_center, src, out=out, stream=stream), img)


def distance_driven_bp(projector: ct_projector, prj, det_center, src, branchless: bool = False, *, out=None,
                       stream=None):
    return D.like_input(D.tomo_bp(projector, prj, det_center, src, out=out, stream=stream), prj)


def filter_fbp(projector: ct_projector, prj, det_center, src, filter_type: str = "hann", cutoff_x: float = 1,
               cutoff_y: float = 1, *, out=None, stream=None, first_view_kernel: bool = False):
    """Tomosynthesis FBP filter (reference tomo.py:157, fbpTomo.cu:50-384):
    each view's rows are filtered with a ramp at the view's virtual pitch
    du * cos(tilt), windowed ('hamming', 'hann', else none) with cut-offs
    ``cutoff_x`` along u and ``cutoff_y`` along the tilt direction (0, 1].
    Returns [batch, nview, nv, nu].  The reference multiplies every view by
    the first view's kernel (fbpTomo.cu:323); ``first_view_kernel=True``
    reproduces that output."""
    return D.like_input(D.tomo_filter(projector, prj, det_center, src, filter_type, cutoff_x, cutoff_y, out=out,
                                      stream=stream, first_view_kernel=first_view_kernel), prj)
