"""Device-array implementation of the projector calls (torch CUDA tensors).

Every function here calls an extended ``ctp_*`` entry of libctp.so on the
caller's (torch current) stream, with the workspace taken from torch's caching
allocator, so a call neither synchronises the device nor calls cudaMalloc once
the allocator is warm.
"""
from __future__ import annotations

from ctypes import byref, c_float, c_ulonglong, c_void_p

import numpy as np
import torch

from .. import _lib
from .._lib import Geometry, check, lib

_LOWP = {torch.bfloat16: (_lib.FLAG_IN_BF16, _lib.FLAG_OUT_BF16), torch.float16: (_lib.FLAG_IN_FP16, _lib.FLAG_OUT_FP16)}
FILTERS = {"hamming": 1, "hann": 2, "cosine": 3}


def filter_code(filter_type: str) -> int:
    """'hamming' 1, 'hann' 2, 'cosine' 3, anything else Ram-Lak 0
    (fan_equiangular.py:39-46 of the reference cupy wrapper)."""
    return FILTERS.get(filter_type.lower(), 0)


def as_tensor(x, lowp_ok: bool = True, dtype=None) -> torch.Tensor:
    """A contiguous CUDA tensor view of x (torch tensor, __cuda_array_interface__
    object, or host array which is uploaded).  Storage dtypes other than
    float32/bfloat16/float16 are cast to float32."""
    if isinstance(x, torch.Tensor):
        t = x
    elif hasattr(x, "__cuda_array_interface__"):
        t = torch.as_tensor(x, device="cuda")
    else:
        t = torch.as_tensor(np.asarray(x))
    if not t.is_cuda:
        t = t.cuda()
    if dtype is not None:
        t = t.to(dtype)
    elif t.dtype == torch.float32 or (lowp_ok and t.dtype in _LOWP):
        pass
    else:
        t = t.float()
    return t.contiguous()


def like_input(out: torch.Tensor, original):
    """Return cupy arrays for cupy inputs (zero copy), torch tensors otherwise."""
    if isinstance(original, torch.Tensor) or not hasattr(original, "__cuda_array_interface__"):
        return out
    try:  # pragma: no cover - cupy is optional
        import cupy

        return cupy.asarray(out)
    except ImportError:  # pragma: no cover
        return out


def ptr(t: torch.Tensor) -> c_void_p:
    return c_void_p(t.data_ptr())


def stream_handle(stream, device) -> c_void_p:
    if stream is None:
        return c_void_p(torch.cuda.current_stream(device).cuda_stream)
    if hasattr(stream, "cuda_stream"):
        return c_void_p(stream.cuda_stream)
    return c_void_p(int(stream))


def workspace(nbytes: int, device):
    if nbytes <= 0:
        return None, c_void_p(0), 0
    ws = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
    return ws, c_void_p(ws.data_ptr()), int(nbytes)


def make_geometry(p, nbatch, image_shape, nu, nv, nview, du, dsd=0.0, dso=0.0) -> Geometry:
    nz, ny, nx = (int(s) for s in image_shape)
    return Geometry(int(nbatch), nx, ny, nz, float(p.dx), float(p.dy), float(p.dz), float(p.cx), float(p.cy),
                    float(p.cz), int(nu), int(nv), int(nview), float(du), float(p.dv), float(p.off_u),
                    float(p.off_v), float(dsd), float(dso))


def fan_da(p) -> float:
    """Angular cell size passed by the reference fan wrappers (du / dsd)."""
    return float(np.float32(p.du / p.dsd))


def _out(shape, dtype, device, out):
    if out is not None:
        if tuple(out.shape) != tuple(shape):
            raise ValueError(f"out has shape {tuple(out.shape)}, expected {tuple(shape)}")
        if not out.is_contiguous():
            raise ValueError("out must be contiguous")
        return out
    return torch.empty(shape, dtype=dtype or torch.float32, device=device)


def _io_flags(inp: torch.Tensor, outp: torch.Tensor) -> int:
    f = 0
    if inp.dtype in _LOWP:
        f |= _LOWP[inp.dtype][0]
    if outp.dtype in _LOWP:
        f |= _LOWP[outp.dtype][1]
    return f


# --------------------------------------------------------------------------- DD 2D
def dd_fp(p, img, angles, geom: int, branchless=False, type_projector: int = 0, out=None, stream=None, dtype=None):
    t = as_tensor(img)
    ang = as_tensor(angles, lowp_ok=False)
    nb = t.shape[0]
    du = fan_da(p) if geom == _lib.GEOM_FAN else float(p.du)
    g = make_geometry(p, nb, t.shape[1:], p.nu, p.nv, ang.numel(), du,
                      *((float(p.dsd), float(p.dso)) if geom == _lib.GEOM_FAN else (1000.0, 500.0)))
    prj = _out([nb, ang.numel(), int(p.nv), int(p.nu)], dtype, t.device, out)
    tp = type_projector | (_lib.TYPE_BRANCHLESS if branchless else 0)
    flags = _io_flags(t, prj)
    ws, wp, wn = workspace(lib().ctp_dd2d_fp_workspace(byref(g), geom, tp, flags), t.device)
    check(lib().ctp_dd2d_fp(ptr(prj), ptr(t), ptr(ang), byref(g), geom, tp, flags, wp, wn,
                            stream_handle(stream, t.device)), "distance_driven_fp")
    return prj


def dd_bp(p, prj, angles, geom: int, is_fbp=False, branchless=False, adjoint=False, type_projector: int = 0,
          out=None, accumulate=False, stream=None, dtype=None):
    t = as_tensor(prj)
    ang = as_tensor(angles, lowp_ok=False)
    nb, nview, nv, nu = t.shape
    du = fan_da(p) if geom == _lib.GEOM_FAN else float(p.du)
    g = make_geometry(p, nb, (p.nz, p.ny, p.nx), nu, nv, nview, du,
                      *((float(p.dsd), float(p.dso)) if geom == _lib.GEOM_FAN else (1000.0, 500.0)))
    img = _out([nb, int(p.nz), int(p.ny), int(p.nx)], dtype, t.device, out)
    tp = type_projector | (_lib.TYPE_FBP if is_fbp else 0) | (_lib.TYPE_BRANCHLESS if branchless else 0)
    flags = _io_flags(t, img) | (0 if accumulate else _lib.FLAG_ZERO_OUT) | (_lib.FLAG_ADJOINT if adjoint else 0)
    ws, wp, wn = workspace(lib().ctp_dd2d_bp_workspace(byref(g), geom, tp, flags), t.device)
    check(lib().ctp_dd2d_bp(ptr(img), ptr(t), ptr(ang), byref(g), geom, tp, flags, wp, wn,
                            stream_handle(stream, t.device)), "distance_driven_bp")
    return img


def dd_nnz(p, angles, geom: int, image_shape=None) -> int:
    """Operator nonzeros of one batch item of the DD forward projector."""
    ang = as_tensor(angles, lowp_ok=False)
    du = fan_da(p) if geom == _lib.GEOM_FAN else float(p.du)
    shape = image_shape if image_shape is not None else (p.nz, p.ny, p.nx)
    g = make_geometry(p, 1, shape, p.nu, p.nv, ang.numel(), du,
                      *((float(p.dsd), float(p.dso)) if geom == _lib.GEOM_FAN else (1000.0, 500.0)))
    n = c_ulonglong(0)
    check(lib().ctp_dd2d_nnz(byref(n), ptr(ang), byref(g), geom, stream_handle(None, ang.device)), "dd2d_nnz")
    return int(n.value)


# --------------------------------------------------------------------------- filters
def ramp_filter(p, prj, filter_type: str, geom: int, out=None, stream=None, exact=False):
    t = as_tensor(prj, lowp_ok=False)
    nb, nview, nv, nu = t.shape
    du = fan_da(p) if geom == _lib.GEOM_FAN else float(p.du)
    g = make_geometry(p, nb, (1, 1, 1), nu, nv, nview, du, float(p.dsd), float(p.dso))
    fprj = _out(list(t.shape), torch.float32, t.device, out)
    ifilter = filter_code(filter_type)
    flags = _lib.FLAG_FILTER_EXACT if exact else 0
    ws, wp, wn = workspace(lib().ctp_ramp_filter_workspace(byref(g), geom, ifilter, flags), t.device)
    check(lib().ctp_ramp_filter(ptr(fprj), ptr(t), byref(g), geom, ifilter, flags, wp, wn,
                                stream_handle(stream, t.device)), "ramp_filter")
    return fprj


def fbp_bp(p, prj, angles, out=None, accumulate=False, stream=None):
    t = as_tensor(prj, lowp_ok=False)
    ang = as_tensor(angles, lowp_ok=False)
    nb, nview, nv, nu = t.shape
    g = make_geometry(p, nb, (p.nz, p.ny, p.nx), nu, nv, nview, fan_da(p), float(p.dsd), float(p.dso))
    img = _out([nb, int(p.nz), int(p.ny), int(p.nx)], torch.float32, t.device, out)
    flags = 0 if accumulate else _lib.FLAG_ZERO_OUT
    check(lib().ctp_fbp_fan_bp(ptr(img), ptr(t), ptr(ang), byref(g), flags, stream_handle(stream, t.device)),
          "fbp_bp")
    return img


# --------------------------------------------------------------------------- Siddon cone
def _geom3(a):
    return as_tensor(a, lowp_ok=False)


def siddon_fp(p, img, det_center, det_u, det_v, src, out=None, accumulate=False, stream=None, dtype=None):
    t = as_tensor(img)
    dc, du_, dv_, sr = _geom3(det_center), _geom3(det_u), _geom3(det_v), _geom3(src)
    nb = t.shape[0]
    nview = dc.shape[0]
    g = make_geometry(p, nb, t.shape[1:], p.nu, p.nv, nview, float(p.du))
    prj = _out([nb, nview, int(p.nv), int(p.nu)], dtype, t.device, out)
    flags = _io_flags(t, prj) | (0 if accumulate else _lib.FLAG_ZERO_OUT)
    check(lib().ctp_siddon_fp(ptr(prj), ptr(t), ptr(dc), ptr(du_), ptr(dv_), ptr(sr), byref(g), flags,
                              stream_handle(stream, t.device)), "siddon_fp_arbitrary")
    return prj


def siddon_bp(p, prj, det_center, det_u, det_v, src, out=None, accumulate=False, stream=None):
    t = as_tensor(prj)
    dc, du_, dv_, sr = _geom3(det_center), _geom3(det_u), _geom3(det_v), _geom3(src)
    nb, nview, nv, nu = t.shape
    g = make_geometry(p, nb, (p.nz, p.ny, p.nx), nu, nv, nview, float(p.du))
    img = _out([nb, int(p.nz), int(p.ny), int(p.nx)], torch.float32, t.device, out)
    flags = _io_flags(t, img) | (0 if accumulate else _lib.FLAG_ZERO_OUT)
    check(lib().ctp_siddon_bp(ptr(img), ptr(t), ptr(dc), ptr(du_), ptr(dv_), ptr(sr), byref(g), flags,
                              stream_handle(stream, t.device)), "siddon_bp_arbitrary")
    return img


def siddon_nnz(p, det_center, det_u, det_v, src, image_shape=None) -> int:
    dc, du_, dv_, sr = _geom3(det_center), _geom3(det_u), _geom3(det_v), _geom3(src)
    shape = image_shape if image_shape is not None else (p.nz, p.ny, p.nx)
    g = make_geometry(p, 1, shape, p.nu, p.nv, dc.shape[0], float(p.du))
    n = c_ulonglong(0)
    check(lib().ctp_siddon_nnz(byref(n), ptr(dc), ptr(du_), ptr(dv_), ptr(sr), byref(g),
                               stream_handle(None, dc.device)), "siddon_nnz")
    return int(n.value)


# --------------------------------------------------------------------------- tomo
def tomo_fp(p, img, det_center, src, out=None, stream=None):
    t = as_tensor(img, lowp_ok=False)
    dc, sr = _geom3(det_center), _geom3(src)
    nb = t.shape[0]
    g = make_geometry(p, nb, t.shape[1:], p.nu, p.nv, dc.shape[0], float(p.du))
    prj = _out([nb, dc.shape[0], int(p.nv), int(p.nu)], torch.float32, t.device, out)
    check(lib().ctp_tomo_fp(ptr(prj), ptr(t), ptr(dc), ptr(sr), byref(g), 0, stream_handle(stream, t.device)),
          "tomo distance_driven_fp")
    return prj


def tomo_bp(p, prj, det_center, src, out=None, stream=None):
    t = as_tensor(prj, lowp_ok=False)
    dc, sr = _geom3(det_center), _geom3(src)
    nb, nview, nv, nu = t.shape
    g = make_geometry(p, nb, (p.nz, p.ny, p.nx), nu, nv, nview, float(p.du))
    img = _out([nb, int(p.nz), int(p.ny), int(p.nx)], torch.float32, t.device, out)
    ws, wp, wn = workspace(lib().ctp_tomo_bp_workspace(byref(g)), t.device)
    check(lib().ctp_tomo_bp(ptr(img), ptr(t), ptr(dc), ptr(sr), byref(g), 0, wp, wn,
                            stream_handle(stream, t.device)), "tomo distance_driven_bp")
    return img


def tomo_filter(p, prj, det_center, src, filter_type: str = "hann", cutoff_x: float = 1.0, cutoff_z: float = 1.0,
                out=None, stream=None, first_view_kernel: bool = False):
    """Tomosynthesis FBP filter; 'hamming' 1, 'hann' 2, anything else none
    (tomo.py:188-193 of the reference cupy wrapper).  ``first_view_kernel``
    filters every view with the first view's kernel, as the reference does."""
    t = as_tensor(prj, lowp_ok=False)
    dc, sr = _geom3(det_center), _geom3(src)
    nb, nview, nv, nu = t.shape
    g = make_geometry(p, nb, (1, 1, 1), nu, nv, nview, float(p.du))
    fprj = _out(list(t.shape), torch.float32, t.device, out)
    ft = filter_type.lower()
    ifilter = 1 if ft == "hamming" else 2 if ft == "hann" else 0
    ws, wp, wn = workspace(lib().ctp_tomo_filter_workspace(byref(g)), t.device)
    flags = _lib.FLAG_TOMO_FIRST_VIEW_KERNEL if first_view_kernel else 0
    check(lib().ctp_tomo_filter(ptr(fprj), ptr(t), ptr(dc), ptr(sr), byref(g), ifilter, c_float(cutoff_x),
                                c_float(cutoff_z), flags, wp, wn, stream_handle(stream, t.device)), "tomo filter_fbp")
    return fprj


# --------------------------------------------------------------------------- numpy-only reference projectors
def siddon_fan_fp(p, img, angles, out=None, stream=None):
    """Fan-beam Siddon forward projection (the reference's numpy siddon_fp)."""
    t = as_tensor(img, lowp_ok=False)
    ang = as_tensor(angles, lowp_ok=False)
    nb = t.shape[0]
    g = make_geometry(p, nb, t.shape[1:], p.nu, p.nv, ang.numel(), fan_da(p), float(p.dsd), float(p.dso))
    prj = _out([nb, ang.numel(), int(p.nv), int(p.nu)], torch.float32, t.device, out)
    check(lib().ctp_siddon_fan_fp(ptr(prj), ptr(t), ptr(ang), byref(g), _lib.FLAG_ZERO_OUT,
                                  stream_handle(stream, t.device)), "siddon_fp")
    return prj


def siddon_fan_bp(p, prj, angles, out=None, accumulate=False, stream=None):
    """Fan-beam Siddon back projection (transpose of siddon_fan_fp)."""
    t = as_tensor(prj, lowp_ok=False)
    ang = as_tensor(angles, lowp_ok=False)
    nb, nview, nv, nu = t.shape
    g = make_geometry(p, nb, (p.nz, p.ny, p.nx), nu, nv, nview, fan_da(p), float(p.dsd), float(p.dso))
    img = _out([nb, int(p.nz), int(p.ny), int(p.nx)], torch.float32, t.device, out)
    check(lib().ctp_siddon_fan_bp(ptr(img), ptr(t), ptr(ang), byref(g), 0 if accumulate else _lib.FLAG_ZERO_OUT,
                                  stream_handle(stream, t.device)), "siddon_bp")
    return img


def pixel_bp_parallel(p, prj, angles, out=None, accumulate=False, stream=None):
    """Pixel-driven parallel back projection (the reference's numpy pixel_driven_bp)."""
    t = as_tensor(prj, lowp_ok=False)
    ang = as_tensor(angles, lowp_ok=False)
    nb, nview, nv, nu = t.shape
    g = make_geometry(p, nb, (p.nz, p.ny, p.nx), nu, nv, nview, float(p.du))
    img = _out([nb, int(p.nz), int(p.ny), int(p.nx)], torch.float32, t.device, out)
    check(lib().ctp_pixel_bp_parallel(ptr(img), ptr(t), ptr(ang), byref(g), 0 if accumulate else _lib.FLAG_ZERO_OUT,
                                      stream_handle(stream, t.device)), "pixel_driven_bp")
    return img

