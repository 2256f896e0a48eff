"""16-bit affine sinogram storage (no counterpart in the reference).

A sinogram [batch, nview, nv, nu] is held as one unsigned 16-bit code per
sample plus, per view of each batch item, an FP32 offset ``lo`` (the view's
minimum) and ``step`` (its range / 65535): value = lo + step * code.  That is
half the bytes of FP32, like BF16 and FP16, but the rounding error is at most
1/131070 of the view's range (3e-5 for line integrals of 0-8), where FP16
rounds a value of 6 by up to 2e-3: reconstructions from it stay within 1e-4 of
the FP32-input ones, which the float formats do not (the ramp filter and the
back projection magnify their rounding).  Codes are kept in int16 tensors
holding the uint16 bit patterns.

All device work runs in libctp.so (csrc/quant.cu; the exact ramp filter reads
the codes directly, csrc/fbp.cu).
"""
from __future__ import annotations

from ctypes import byref
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from ._lib import check, lib
from .projector import _device as D


@dataclass
class Q16:
    """A sinogram in 16-bit affine storage: ``code`` int16 [..., nview, nv, nu]
    (uint16 bit patterns), ``lo`` and ``step`` float32 [..., nview]."""

    code: torch.Tensor
    lo: torch.Tensor
    step: torch.Tensor

    @property
    def shape(self):
        return self.code.shape

    @property
    def device(self):
        return self.code.device

    @property
    def nbytes(self) -> int:
        return self.code.numel() * 2 + (self.lo.numel() + self.step.numel()) * 4

    def __getitem__(self, key) -> "Q16":
        """Slices along the batch dimension."""
        return Q16(self.code[key], self.lo[key], self.step[key])

    def pin_memory(self) -> "Q16":
        return Q16(self.code.pin_memory(), self.lo.pin_memory(), self.step.pin_memory())

    def to(self, device, non_blocking: bool = False) -> "Q16":
        return Q16(self.code.to(device, non_blocking=non_blocking), self.lo.to(device, non_blocking=non_blocking),
                   self.step.to(device, non_blocking=non_blocking))

    def cpu(self) -> "Q16":
        return self.to("cpu")

    def float(self) -> torch.Tensor:
        """The stored values as float32 on the code's device (on the host:
        computed in FP64 and rounded once, within one FP32 rounding of the
        kernels' fused multiply-add)."""
        if self.code.is_cuda:
            return dequantize(self)
        codes = self.code.to(torch.int32) & 0xFFFF
        lo = self.lo.reshape(*self.lo.shape, 1, 1)
        step = self.step.reshape(*self.step.shape, 1, 1)
        return (lo.double() + step.double() * codes.double()).float()


def _rows(shape):
    *lead, nv, nu = shape
    nrows = 1
    for s in lead:
        nrows *= int(s)
    return nrows, int(nv) * int(nu)


def quantize(y: torch.Tensor, stream=None) -> Q16:
    """Quantize a float32 CUDA sinogram [..., nview, nv, nu]: one offset and step
    per view."""
    if not (y.is_cuda and y.dtype == torch.float32):
        raise TypeError("quantize takes a float32 CUDA tensor")
    y = y.contiguous()
    nrows, row_len = _rows(y.shape)
    code = torch.empty(y.shape, dtype=torch.int16, device=y.device)
    lo = torch.empty(y.shape[:-2], dtype=torch.float32, device=y.device)
    step = torch.empty(y.shape[:-2], dtype=torch.float32, device=y.device)
    check(lib().ctp_quantize_u16(D.ptr(code), D.ptr(lo), D.ptr(step), D.ptr(y), nrows, row_len,
                                 D.stream_handle(stream, y.device)), "quantize_u16")
    return Q16(code, lo, step)


def dequantize(q: Q16, out: Optional[torch.Tensor] = None, subtract: bool = False, stream=None) -> torch.Tensor:
    """float32 values of ``q`` (into ``out``), or ``out -= values`` with
    subtract=True (the SQS residual A x - y)."""
    nrows, row_len = _rows(q.shape)
    if out is None:
        if subtract:
            raise ValueError("subtract needs out")
        out = torch.empty(q.shape, dtype=torch.float32, device=q.device)
    if tuple(out.shape) != tuple(q.shape) or not out.is_contiguous():
        raise ValueError("out must be a contiguous tensor of the sinogram's shape")
    check(lib().ctp_dequantize_u16(D.ptr(out), D.ptr(q.code), D.ptr(q.lo), D.ptr(q.step), nrows, row_len,
                                   _lib.FLAG_SUBTRACT if subtract else 0, D.stream_handle(stream, out.device)),
          "dequantize_u16")
    return out


def sub_dequantized_(r: torch.Tensor, q: Q16, stream=None) -> torch.Tensor:
    """r -= the values of q, in place."""
    return dequantize(q, out=r, subtract=True, stream=stream)


def ramp_filter(p, q: Q16, filter_type: str, geom: int, out=None, stream=None) -> torch.Tensor:
    """The exact (FP64) ramp filter of a sinogram in 16-bit affine storage;
    geom 0 fan, 1 parallel (as projector._device.ramp_filter)."""
    nb, nview, nv, nu = (int(s) for s in q.shape)
    du = D.fan_da(p) if geom == _lib.GEOM_FAN else float(p.du)
    g = D.make_geometry(p, nb, (1, 1, 1), nu, nv, nview, du, float(p.dsd), float(p.dso))
    fprj = D._out([nb, nview, nv, nu], torch.float32, q.device, out)
    check(lib().ctp_ramp_filter_u16(D.ptr(fprj), D.ptr(q.code), D.ptr(q.lo), D.ptr(q.step), byref(g), geom,
                                    D.filter_code(filter_type), D.stream_handle(stream, q.device)),
          "ramp_filter_u16")
    return fprj


__all__ = ["Q16", "quantize", "dequantize", "sub_dequantized_", "ramp_filter"]
