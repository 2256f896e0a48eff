"""Cone-beam arbitrary trajectory (Siddon), host arrays.

Same calls as ct_projector/projector/numpy/cone.py of the reference:
siddon_fp_arbitrary (:19), siddon_bp_arbitrary (:96).
"""
from __future__ import annotations

import numpy as np

from ._host import c_float, call, f32, geom_args, out_array, p
from .ct_projector import ct_projector


def siddon_fp_arbitrary(projector: ct_projector, img, det_center, det_u, det_v, src) -> np.ndarray:
    img, det_center, det_u, det_v, src = (f32(a) for a in (img, det_center, det_u, det_v, src))
    prj = out_array([img.shape[0], det_center.shape[0], projector.nv, projector.nu])
    call("cSiddonConeProjectionArbitrary", p(prj), p(img), p(det_center), p(det_u), p(det_v), p(src),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:]), c_float(projector.du),
         c_float(projector.dv), c_float(projector.off_u), c_float(projector.off_v))
    return prj


def siddon_bp_arbitrary(projector: ct_projector, prj, det_center, det_u, det_v, src) -> np.ndarray:
    prj, det_center, det_u, det_v, src = (f32(a) for a in (prj, det_center, det_u, det_v, src))
    img = out_array([prj.shape[0], projector.nz, projector.ny, projector.nx])
    call("cSiddonConeBackprojectionArbitrary", p(img), p(prj), p(det_center), p(det_u), p(det_v), p(src),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:]), c_float(projector.du),
         c_float(projector.dv), c_float(projector.off_u), c_float(projector.off_v))
    return img
