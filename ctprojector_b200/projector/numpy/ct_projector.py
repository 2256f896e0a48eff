"""ct_projector for host arrays (reference ct_projector/projector/numpy/ct_projector.py)."""
from __future__ import annotations

import numpy as np

from ..._lib import lib
from ...geometry import ct_projector_base


def set_device(device: int) -> int:
    """Set the computing device and return any error code."""
    return lib().SetDevice(int(device))


class ct_projector(ct_projector_base):
    """CT projector wrapper; power-method helpers in numpy."""

    def _rand(self, shape):
        return np.random.uniform(size=shape).astype(np.float32)

    def _ones(self, shape):
        return np.ones(shape, dtype=np.float32)

    def _norm(self, x) -> float:
        return float(np.linalg.norm(x))

    def _sqrt(self, x):
        return np.sqrt(x)
