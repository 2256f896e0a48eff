"""Cone-beam arbitrary trajectory (Siddon), device arrays.

Same calls as ct_projector/projector/cupy/cone.py of the reference:
siddon_fp_arbitrary (:15), siddon_bp_arbitrary (:87).  Geometry arrays are
[nview, 3] as (x, y, z) in mm (siddonCone.cu:36-37 reads float3 {x, y, z}).
"""
from __future__ import annotations

from .. import _device as D
from .ct_projector import ct_projector


def siddon_fp_arbitrary(projector: ct_projector, img, det_center, det_u, det_v, src, *, out=None,
                        accumulate=False, stream=None, dtype=None):
    """Forward projection; image size from img, detector from projector.nu/nv."""
    return D.like_input(D.siddon_fp(projector, img, det_center, det_u, det_v, src, out=out, accumulate=accumulate,
                                    stream=stream, dtype=dtype), img)


def siddon_bp_arbitrary(projector: ct_projector, prj, det_center, det_u, det_v, src, *, out=None, accumulate=False,
                        stream=None):
    """Back projection (transpose of siddon_fp_arbitrary); image size from projector."""
    return D.like_input(D.siddon_bp(projector, prj, det_center, det_u, det_v, src, out=out, accumulate=accumulate,
                                    stream=stream), prj)
