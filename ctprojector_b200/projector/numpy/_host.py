"""Shared helpers of the host-array modules: float32 C-contiguous buffers and
the reference argument lists of the c* entries."""
from __future__ import annotations

from ctypes import c_float, c_int, c_size_t, c_void_p

import numpy as np

from ..._lib import check, lib


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def p(a: np.ndarray) -> c_void_p:
    return c_void_p(a.ctypes.data)


def geom_args(proj, nb, image_shape, prj_shape):
    """nBatches, nx, ny, nz, dx, dy, dz, cx, cy, cz, nu, nv, nview."""
    nz, ny, nx = image_shape
    nview, nv, nu = prj_shape
    return [c_size_t(int(nb)), c_size_t(int(nx)), c_size_t(int(ny)), c_size_t(int(nz)), c_float(proj.dx),
            c_float(proj.dy), c_float(proj.dz), c_float(proj.cx), c_float(proj.cy), c_float(proj.cz),
            c_size_t(int(nu)), c_size_t(int(nv)), c_size_t(int(nview))]


def call(name: str, *args):
    check(getattr(lib(), name)(*args), name)


__all__ = ["f32", "p", "geom_args", "call", "c_float", "c_int", "c_size_t"]
