"""Shared helpers of the host-array modules: float32 C-contiguous buffers and
the reference argument lists of the c* entries."""
from __future__ import annotations

import ctypes
from ctypes import c_float, c_int, c_size_t, c_void_p

import numpy as np

from ..._lib import check, lib

_HUGE = 2 << 20  # transparent huge page
_MADV_HUGEPAGE = 14
try:
    _madvise = ctypes.CDLL(None, use_errno=True).madvise
    _madvise.argtypes = [c_void_p, c_size_t, c_int]
    _madvise.restype = c_int
except (OSError, AttributeError):
    _madvise = None

# Output arrays of at least 8 MB are backed by transparent huge pages where
# the kernel offers them (module switch, on by default).
huge_outputs = True


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def out_array(shape) -> np.ndarray:
    """A float32 output array for a host entry, which overwrites all of it.
    The first write of a fresh array costs a page fault and a page clear per
    4 KB page; large arrays are advised onto 2 MB pages (madvise
    MADV_HUGEPAGE), which takes 512 times fewer faults."""
    n = int(np.prod(shape)) * 4
    if not huge_outputs or _madvise is None or n < 4 * _HUGE:
        return np.empty(shape, np.float32)
    buf = np.empty(n + _HUGE, np.uint8)
    off = (-buf.ctypes.data) % _HUGE
    _madvise(c_void_p(buf.ctypes.data + off), c_size_t(n // _HUGE * _HUGE), _MADV_HUGEPAGE)  # a hint: failure is harmless
    return buf[off:off + n].view(np.float32).reshape(shape)


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


def exact_filter(projector, prj: np.ndarray, filter_type: str, geom: int, du: float) -> np.ndarray:
    """The FP64 ramp filter (ctp_ramp_filter_host with CTP_FLAG_FILTER_EXACT)
    on a float32 host sinogram; du is the cell size the reference passes
    (angular for fan beams)."""
    from ..._lib import FLAG_FILTER_EXACT, Geometry
    from .._device import filter_code

    nb, nview, nv, nu = prj.shape
    g = Geometry(nb, 1, 1, 1, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, nu, nv, nview, float(du), float(projector.dv),
                 float(projector.off_u), float(projector.off_v), float(getattr(projector, "dsd", 0.0)),
                 float(getattr(projector, "dso", 0.0)))
    fprj = out_array(prj.shape)
    call("ctp_ramp_filter_host", p(fprj), p(prj), ctypes.byref(g), geom, filter_code(filter_type), FLAG_FILTER_EXACT)
    return fprj


__all__ = ["f32", "out_array", "p", "geom_args", "call", "exact_filter", "c_float", "c_int", "c_size_t"]
