"""ct_projector for device arrays (reference ct_projector/projector/cupy/ct_projector.py)."""
from __future__ import annotations

import torch

from ..._lib import lib
from ...geometry import ct_projector_base


def set_device(device: int) -> int:
    """Set the computing device and return any error code (ct_projector.py:20-24)."""
    torch.cuda.set_device(device)
    return lib().SetDevice(int(device))


class ct_projector(ct_projector_base):
    """CT projector wrapper; power-method helpers run on the current CUDA device."""

    def _rand(self, shape):
        return torch.rand(shape, dtype=torch.float32, device="cuda")

    def _ones(self, shape):
        return torch.ones(shape, dtype=torch.float32, device="cuda")

    def _norm(self, x) -> float:
        return float(torch.linalg.vector_norm(x.float()))

    def _sqrt(self, x):
        return torch.sqrt(x)
