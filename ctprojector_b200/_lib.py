"""ctypes binding of libctp.so (the sm_100a kernels and C ABI, include/ctp.h).

The library is built in-tree by ``python -m ctprojector_b200.build``.  There is
no CPU fallback: if the library is missing or fails to load, every projector
call raises ``CTProjectorError``.
"""
from __future__ import annotations

import ctypes
import os
import threading
from ctypes import POINTER, Structure, c_char_p, c_float, c_int, c_size_t, c_uint, c_ulonglong, c_void_p

from .errors import CTProjectorError

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libctp.so")

# status codes and flags, include/ctp.h
CTP_OK = 0
CTP_ERR_INVALID_ARGUMENT = 1001
CTP_ERR_UNSUPPORTED = 1002
CTP_ERR_WORKSPACE = 1003
CTP_ERR_CUFFT = 1004
CTP_ERR_TOO_LARGE = 1005
CTP_ERR_WAIT_TIMEOUT = 1006
CTP_WAIT_POLLS_DEFAULT = 4194304

FLAG_ZERO_OUT = 0x1
FLAG_ADJOINT = 0x2
FLAG_IN_BF16 = 0x10
FLAG_IN_FP16 = 0x20
FLAG_OUT_BF16 = 0x40
FLAG_OUT_FP16 = 0x80
FLAG_FILTER_EXACT = 0x100
FLAG_SUBTRACT = 0x400
FLAG_TOMO_FIRST_VIEW_KERNEL = 0x200

TYPE_FBP = 0x1
TYPE_BRANCHLESS = 0x2
TYPE_FORCE_FBP = 0x4

GEOM_FAN = 0
GEOM_PARALLEL = 1


class Geometry(Structure):
    """ctp_geometry (include/ctp.h)."""

    _fields_ = [("nbatch", c_size_t), ("nx", c_size_t), ("ny", c_size_t), ("nz", c_size_t),
                ("dx", c_float), ("dy", c_float), ("dz", c_float),
                ("cx", c_float), ("cy", c_float), ("cz", c_float),
                ("nu", c_size_t), ("nv", c_size_t), ("nview", c_size_t),
                ("du", c_float), ("dv", c_float), ("off_u", c_float), ("off_v", c_float),
                ("dsd", c_float), ("dso", c_float)]


_lock = threading.Lock()
_lib = None

_P = c_void_p
_F = c_float
_S = c_size_t
_GP = POINTER(Geometry)
_REF_GEOM = [_S, _S, _S, _S, _F, _F, _F, _F, _F, _F, _S, _S, _S]  # nBatches, nx..cz, nu, nv, nview

# name -> argtypes; every entry returns int unless listed in _RESTYPE
_SIGNATURES = {
    "SetDevice": [c_int],
    "cupyDistanceDrivenFanProjection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, _F, _F, c_int],
    "cDistanceDrivenFanProjection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, _F, _F, c_int],
    "cupyDistanceDrivenParallelProjection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "cDistanceDrivenParallelProjection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "cupyDistanceDrivenFanBackprojection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, _F, _F, c_int],
    "cDistanceDrivenFanBackprojection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, _F, _F, c_int],
    "cupyDistanceDrivenParallelBackprojection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "cDistanceDrivenParallelBackprojection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "cupyDistanceDrivenTomoProjection": [_P, _P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "cDistanceDrivenTomoProjection": [_P, _P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "cupyDistanceDrivenTomoBackprojection": [_P, _P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "cDistanceDrivenTomoBackprojection": [_P, _P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "cupySiddonConeProjectionArbitrary": [_P, _P, _P, _P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F],
    "cSiddonConeProjectionArbitrary": [_P, _P, _P, _P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F],
    "cupySiddonConeBackprojectionArbitrary": [_P, _P, _P, _P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F],
    "cSiddonConeBackprojectionArbitrary": [_P, _P, _P, _P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F],
    "cupyfbpFanFilter": [_P, _P, c_int, _S, _S, _S, _F, _F, _F, _F, _F, _F, c_int],
    "cfbpFanFilter": [_P, _P, c_int, _S, _S, _S, _F, _F, _F, _F, _F, _F, c_int],
    "cupyfbpParallelFilter": [_P, _P, c_int, _S, _S, _S, _F, _F, _F, _F, c_int],
    "cfbpParallelFilter": [_P, _P, c_int, _S, _S, _S, _F, _F, _F, _F, c_int],
    "cupyfbpFanBackprojection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, _F, _F],
    "cfbpFanBackprojection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, _F, _F],
    "ctpGetLastErrorString": [],
    "ctpVersion": [],
    "ctp_dd2d_fp": [_P, _P, _P, _GP, c_int, c_int, c_uint, _P, _S, _P],
    "ctp_dd2d_fp_workspace": [_GP, c_int, c_int, c_uint],
    "ctp_dd2d_bp": [_P, _P, _P, _GP, c_int, c_int, c_uint, _P, _S, _P],
    "ctp_dd2d_bp_workspace": [_GP, c_int, c_int, c_uint],
    "ctp_dd2d_nnz": [POINTER(c_ulonglong), _P, _GP, c_int, _P],
    "ctp_dd2d_fp_noalloc": [_P, _P, _P, _GP, c_int, c_int, c_uint, _P],
    "ctp_dd2d_fp_noalloc_capacity": [],
    "ctp_ramp_filter": [_P, _P, _GP, c_int, c_int, c_uint, _P, _S, _P],
    "ctp_ramp_filter_workspace": [_GP, c_int, c_int, c_uint],
    "ctp_fbp_fan_bp": [_P, _P, _P, _GP, c_uint, _P],
    "ctp_siddon_fp": [_P, _P, _P, _P, _P, _P, _GP, c_uint, _P],
    "ctp_siddon_bp": [_P, _P, _P, _P, _P, _P, _GP, c_uint, _P],
    "ctp_siddon_nnz": [POINTER(c_ulonglong), _P, _P, _P, _P, _GP, _P],
    "ctp_tomo_fp": [_P, _P, _P, _P, _GP, c_uint, _P],
    "ctp_tomo_bp": [_P, _P, _P, _P, _GP, c_uint, _P, _S, _P],
    "ctp_tomo_bp_workspace": [_GP],
    "cupyTVSQS3D": [_P, _P, _P, _P, _F, _F, _F, _S, _S, _S, _S, _F],
    "cTVSQS3D": [_P, _P, _P, _P, _F, _F, _F, _S, _S, _S, _S, _F],
    "ctp_tv_sqs": [_P, _P, _P, _P, _F, _F, _F, _S, _S, _S, _S, _F, _P],
    "ctp_wait_timeouts": [_P],
    "ctp_ramp_filter_host": [_P, _P, _GP, c_int, c_int, c_uint],
    "ctp_quantize_u16": [_P, _P, _P, _P, _S, _S, _P],
    "ctp_dequantize_u16": [_P, _P, _P, _P, _S, _S, c_uint, _P],
    "ctp_ramp_filter_u16": [_P, _P, _P, _P, _GP, c_int, c_int, _P],
    "ctp_set_wait_limit": [c_uint],
    "ctp_set_fp_stream_slices": [c_int],
    "ctp_scratch_allocations": [_P],
    "cSiddonFanProjection": [_P, _P, _P, c_int, _S, _S, _S, _F, _F, _F, _F, _F, _F, _S, _S, _S, _F, _F, _F, _F, _F, _F],
    "cSiddonFanBackprojection": [_P, _P, _P, c_int, _S, _S, _S, _F, _F, _F, _F, _F, _F, _S, _S, _S, _F, _F, _F, _F, _F,
                                 _F],
    "cfbpParallelBackprojection": [_P, _P, _P] + _REF_GEOM + [_F, _F, _F, _F, c_int],
    "ctp_siddon_fan_fp": [_P, _P, _P, _GP, c_uint, _P],
    "ctp_siddon_fan_bp": [_P, _P, _P, _GP, c_uint, _P],
    "ctp_pixel_bp_parallel": [_P, _P, _P, _GP, c_uint, _P],
    "cupyFbpTomoFilter": [_P, _P, _P, _P, c_int, _S, _S, _S, _F, _F, _F, c_int, _F, _F],
    "ctp_tomo_filter": [_P, _P, _P, _P, _GP, c_int, _F, _F, c_uint, _P, _S, _P],
    "ctp_tomo_filter_workspace": [_GP],
    "ctp_sqs_tv_update": [_P, _P, _P, _P, _P, _S, _P, _F, _F, _F, _F, _F, _S, _S, _S, c_uint, _P],
}
_RESTYPE = {
    "ctpGetLastErrorString": c_char_p,
    "ctpVersion": c_char_p,
    "ctp_dd2d_fp_workspace": c_size_t,
    "ctp_tomo_filter_workspace": c_size_t,
    "ctp_dd2d_bp_workspace": c_size_t,
    "ctp_dd2d_fp_noalloc_capacity": c_size_t,
    "ctp_ramp_filter_workspace": c_size_t,
    "ctp_tomo_bp_workspace": c_size_t,
}


def lib():
    """The loaded libctp.so with argument types set; raises if unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise CTProjectorError(
                    CTP_ERR_UNSUPPORTED,
                    f"CUDA extension {LIB_PATH} is not built; run `python -m ctprojector_b200.build` "
                    "(there is no CPU fallback)")
            try:
                L = ctypes.CDLL(LIB_PATH)
            except OSError as e:  # pragma: no cover - depends on the machine
                raise CTProjectorError(CTP_ERR_UNSUPPORTED, f"cannot load {LIB_PATH}: {e}") from e
            for name, args in _SIGNATURES.items():
                f = getattr(L, name)
                f.argtypes = args
                f.restype = _RESTYPE.get(name, c_int)
            _lib = L
    return _lib


def declared_symbols():
    return list(_SIGNATURES)


def last_error_string() -> str:
    s = lib().ctpGetLastErrorString()
    return s.decode() if s else ""


def check(code: int, what: str):
    """Map a status code to CTProjectorError (or print it in non-strict mode)."""
    from . import errors

    if code == 0:
        return
    msg = f"{what} failed with status {code}: {last_error_string()}"
    if errors.is_strict():
        raise CTProjectorError(code, msg)
    print(code)
