"""Equiangular fan-beam geometry, host arrays.

Same calls and module name (sic) as ct_projector/projector/numpy/fan_equiangluar.py
of the reference: ramp_filter (:19), fbp_bp (:75), siddon_fp (:131),
siddon_bp (:185), distance_driven_fp (:241), distance_driven_bp (:302).  Inputs are cast to float32.
"""
from __future__ import annotations

from typing import Union

import numpy as np

from .._device import filter_code
from ._host import c_float, c_int, c_size_t, call, exact_filter, f32, geom_args, out_array, p
from .ct_projector import ct_projector


def ramp_filter(projector: ct_projector, prj: np.ndarray, filter_type: str = "hann", *,
                exact: bool = False) -> np.ndarray:
    """Default: the reference's FP32 filter construction (its rounding
    reproduced); exact=True: the FP64 filter (one-launch FFT convolution)."""
    prj = f32(prj)
    if exact:
        return exact_filter(projector, prj, filter_type, 0, np.float32(projector.du / projector.dsd))
    fprj = out_array(prj.shape)
    call("cfbpFanFilter", p(fprj), p(prj), c_int(prj.shape[0]), c_size_t(prj.shape[3]), c_size_t(prj.shape[2]),
         c_size_t(prj.shape[1]),
         c_float(projector.du / projector.dsd), c_float(projector.dv), c_float(projector.off_u),
         c_float(projector.off_v), c_float(projector.dsd), c_float(projector.dso), c_int(filter_code(filter_type)))
    return fprj


def fbp_bp(projector: ct_projector, prj: np.ndarray, angles: np.ndarray) -> np.ndarray:
    prj = f32(prj)
    angles = f32(angles)
    img = out_array([prj.shape[0], projector.nz, projector.ny, projector.nx])
    call("cfbpFanBackprojection", p(img), p(prj), p(angles),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:]),
         c_float(projector.du / projector.dsd), c_float(projector.dv), c_float(projector.off_u),
         c_float(projector.off_v), c_float(projector.dsd), c_float(projector.dso))
    return img


def distance_driven_fp(projector: ct_projector, img: np.ndarray, angles: np.ndarray,
                       branchless: Union[bool, int] = False) -> np.ndarray:
    img = f32(img)
    angles = f32(angles)
    prj = out_array([img.shape[0], len(angles), projector.nv, projector.nu])
    call("cDistanceDrivenFanProjection", p(prj), p(img), p(angles),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:]),
         c_float(projector.du / projector.dsd), c_float(projector.dv), c_float(projector.off_u),
         c_float(projector.off_v), c_float(projector.dsd), c_float(projector.dso), c_int(2 if branchless else 0))
    return prj


def distance_driven_bp(projector: ct_projector, prj: np.ndarray, angles: np.ndarray,
                       is_fbp: Union[bool, int] = False, branchless: Union[bool, int] = False) -> np.ndarray:
    prj = f32(prj)
    angles = f32(angles)
    img = out_array([prj.shape[0], projector.nz, projector.ny, projector.nx])
    call("cDistanceDrivenFanBackprojection", p(img), p(prj), p(angles),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:]),
         c_float(projector.du / projector.dsd), c_float(projector.dv), c_float(projector.off_u),
         c_float(projector.off_v), c_float(projector.dsd), c_float(projector.dso),
         c_int((1 if is_fbp else 0) + (2 if branchless else 0)))
    return img


def siddon_fp(projector: ct_projector, img: np.ndarray, angles: np.ndarray) -> np.ndarray:
    """Fan-beam forward projection, Siddon ray driven (reference :131)."""
    img = f32(img)
    angles = f32(angles)
    prj = out_array([img.shape[0], len(angles), projector.nv, projector.nu])
    call("cSiddonFanProjection", p(prj), p(img), p(angles), c_int(img.shape[0]),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:])[1:],
         c_float(projector.du / projector.dsd), c_float(projector.dv), c_float(projector.off_u),
         c_float(projector.off_v), c_float(projector.dsd), c_float(projector.dso))
    return prj


def siddon_bp(projector: ct_projector, prj: np.ndarray, angles: np.ndarray) -> np.ndarray:
    """Fan-beam back projection, Siddon ray driven: the transpose of siddon_fp (reference :185)."""
    prj = f32(prj)
    angles = f32(angles)
    img = out_array([prj.shape[0], projector.nz, projector.ny, projector.nx])
    call("cSiddonFanBackprojection", p(img), p(prj), p(angles), c_int(prj.shape[0]),
         *geom_args(projector, img.shape[0], img.shape[1:], prj.shape[1:])[1:],
         c_float(projector.du / projector.dsd), c_float(projector.dv), c_float(projector.off_u),
         c_float(projector.off_v), c_float(projector.dsd), c_float(projector.dso))
    return img
