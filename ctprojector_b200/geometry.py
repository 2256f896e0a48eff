"""The ``ct_projector`` geometry/plug-in class shared by both array back ends.

Mirrors ct_projector/projector/{cupy,numpy}/ct_projector.py:27-195 of the
reference: geometry attributes with the same defaults, ``from_file`` reading a
``[geometry]`` section (keys ending in ``_mm`` lose the suffix, values are cast
to float32, ``n*`` recast to int), the ``set_projector``/``set_backprojector``
plug-in with keyword defaults merged into ``fp``/``bp``, the power-method
``calc_projector_norm``, ``calc_norm_img`` and ``get_angles``.
"""
from __future__ import annotations

import configparser
from typing import Any, Callable

import numpy as np


class ct_projector_base:
    """Geometry container and FP/BP plug-in point (reference ct_projector.py:27)."""

    def __init__(self):
        self.nview = 720
        self.rotview = 720
        self.nu = 512
        self.nv = 512
        self.nx = 512
        self.ny = 512
        self.nz = 512
        self.dx = 1
        self.dy = 1
        self.dz = 1
        self.cx = 0
        self.cy = 0
        self.cz = 0
        self.dsd = 1085.6
        self.dso = 595
        self.du = 1.2
        self.dv = 1.2
        self.off_u = 0
        self.off_v = 0
        self.fp_kwargs: dict = {}
        self.bp_kwargs: dict = {}

    def from_file(self, filename: str) -> None:
        """Load the geometry from a config file (ct_projector.py:52-70)."""
        self.geometry = configparser.ConfigParser()
        _ = self.geometry.read(filename)
        for o in self.geometry["geometry"]:
            if "_mm" in o:
                setattr(self, o[:-3], np.float32(self.geometry["geometry"][o]))
            else:
                setattr(self, o, np.float32(self.geometry["geometry"][o]))
        self.nview = int(self.nview)
        self.nu = int(self.nu)
        self.nv = int(self.nv)
        self.nx = int(self.nx)
        self.ny = int(self.ny)
        self.nz = int(self.nz)

    def set_projector(self, projector: Callable[..., Any], **kwargs) -> None:
        """Register the forward projector called as projector(self, img, **kwargs)."""
        self.projector = projector
        self.fp_kwargs = kwargs

    def set_backprojector(self, backprojector: Callable[..., Any], **kwargs) -> None:
        """Register the back projector called as backprojector(self, prj, **kwargs)."""
        self.backprojector = backprojector
        self.bp_kwargs = kwargs

    def fp(self, img, **kwargs):
        for k in self.fp_kwargs:
            if k not in kwargs:
                kwargs[k] = self.fp_kwargs[k]
        return self.projector(self, img, **kwargs)

    def bp(self, prj, **kwargs):
        for k in self.bp_kwargs:
            if k not in kwargs:
                kwargs[k] = self.bp_kwargs[k]
        return self.backprojector(self, prj, **kwargs)

    def get_angles(self) -> np.ndarray:
        """Angles of a circular scan, 2*pi*i/nview (ct_projector.py:191-195)."""
        return np.arange(0, self.nview, dtype=np.float32) * 2 * np.pi / self.nview

    # array-module specific pieces
    def _rand(self, shape):  # pragma: no cover - overridden
        raise NotImplementedError

    def _ones(self, shape):  # pragma: no cover - overridden
        raise NotImplementedError

    def _norm(self, x) -> float:  # pragma: no cover - overridden
        raise NotImplementedError

    def _sqrt(self, x):  # pragma: no cover - overridden
        raise NotImplementedError

    def calc_projector_norm(self, weight=None, niter: int = 10) -> float:
        """Power method for ||A|| (or ||sqrt(w) A||), ct_projector.py:136-169."""
        weight = self._sqrt(weight) if weight is not None else 1
        x = self._rand([1, self.nz, self.ny, self.nx])
        x = x / self._norm(x)
        norm = 0.0
        for i in range(niter):
            print(i, end=",", flush=True)
            fp = self.fp(x)
            norm = self._norm(fp)
            x = self.bp(fp * weight)
            x = x / self._norm(x)
        print("")
        return norm

    def calc_norm_img(self, weight=None):
        """norm_img = A^T w A 1 (ct_projector.py:171-189)."""
        if weight is None:
            weight = 1
        x = self._ones([1, self.nz, self.ny, self.nx])
        return self.bp(self.fp(x) * weight)
