"""Tomosynthesis geometry, host arrays.

Same calls as ct_projector/projector/numpy/tomo.py of the reference:
distance_driven_fp (:19), distance_driven_bp (:93).
"""
from __future__ import annotations

import numpy as np

from ._host import c_float, c_int, call, f32, geom_args, out_array, p
from .ct_projector import ct_projector


def distance_driven_fp(projector: ct_projector, img, det_center, src, branchless: bool = False) -> np.ndarray:
    img, det_center, src = f32(img), f32(det_center), f32(src)
    prj = out_array([img.shape[0], det_center.shape[0], projector.nv, projector.nu])
    call("cDistanceDrivenTomoProjection", p(prj), p(img), p(det_center), p(src),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:]), c_float(projector.du),
         c_float(projector.dv), c_float(projector.off_u), c_float(projector.off_v), c_int(1 if branchless else 0))
    return prj


def distance_driven_bp(projector: ct_projector, prj, det_center, src, branchless: bool = False) -> np.ndarray:
    prj, det_center, src = f32(prj), f32(det_center), f32(src)
    img = out_array([prj.shape[0], projector.nz, projector.ny, projector.nx])
    call("cDistanceDrivenTomoBackprojection", p(img), p(prj), p(det_center), p(src),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:]), c_float(projector.du),
         c_float(projector.dv), c_float(projector.off_u), c_float(projector.off_v), c_int(1 if branchless else 0))
    return img
