"""Small seeded cases shared by the golden-fixture generator and the tests.

Each case names a geometry (the attributes of the reference ct_projector
class), its seeded inputs and the reference operations recorded for it.
"""
from __future__ import annotations

import numpy as np

from ctprojector_b200 import synthetic as S


class Proj:
    """Plain attribute bag with the reference ct_projector attribute names."""

    def __init__(self, **kw):
        self.nx = self.ny = self.nz = 1
        self.dx = self.dy = self.dz = 1.0
        self.cx = self.cy = self.cz = 0.0
        self.nu = self.nv = 1
        self.du = self.dv = 1.0
        self.off_u = self.off_v = 0.0
        self.dsd = 1085.6
        self.dso = 595.0
        self.nview = 1
        for k, v in kw.items():
            setattr(self, k, v)

    def as_dict(self):
        return {k: v for k, v in self.__dict__.items()}


def _phantom_stack(rng, nb, nz, ny, nx, dx, dy):
    img = np.zeros((nb, nz, ny, nx), np.float32)
    for b in range(nb):
        for z in range(nz):
            img[b, z] = S.ellipse_phantom(rng, nx, ny, dx, dy, supersample=2)
    return img


def case_fan_basic():
    p = Proj(nx=64, ny=64, nz=1, dx=1.0, dy=1.0, nu=96, nv=1, du=1.2858, dv=1.0, nview=90)
    rng = np.random.default_rng(S.seed_for(101))
    ang = S.angles(90, 2 * np.pi)
    img = _phantom_stack(rng, 2, 1, 64, 64, 1.0, 1.0)
    return "fan_basic", p, dict(img=img, angles=ang)


def case_fan_offsets():
    p = Proj(nx=48, ny=56, nz=3, dx=1.1, dy=0.9, dz=1.0, cx=2.5, cy=-1.5, cz=0.0, nu=80, nv=3, du=1.2858, dv=1.0,
             off_u=0.37, off_v=0.3, nview=64)
    rng = np.random.default_rng(S.seed_for(102))
    ang = (np.sort(rng.uniform(0, 2 * np.pi, 64))).astype(np.float32)
    img = _phantom_stack(rng, 1, 3, 56, 48, 1.1, 0.9)
    return "fan_offsets", p, dict(img=img, angles=ang)


def case_par_basic():
    p = Proj(nx=64, ny=64, nz=1, dx=0.8, dy=0.8, nu=96, nv=1, du=0.8, dv=1.0, nview=90)
    rng = np.random.default_rng(S.seed_for(103))
    ang = S.angles(90, np.pi)
    img = _phantom_stack(rng, 2, 1, 64, 64, 0.8, 0.8)
    return "par_basic", p, dict(img=img, angles=ang)


def case_par_offsets():
    p = Proj(nx=40, ny=52, nz=2, dx=1.0, dy=1.2, dz=1.0, cx=-3.0, cy=1.0, nu=72, nv=2, du=0.7, dv=1.0,
             off_u=-0.6, off_v=0.0, nview=50)
    rng = np.random.default_rng(S.seed_for(104))
    ang = (np.sort(rng.uniform(0, np.pi, 50))).astype(np.float32)
    img = _phantom_stack(rng, 1, 2, 52, 40, 1.0, 1.2)
    return "par_offsets", p, dict(img=img, angles=ang)


def case_kat():
    """example/ex_dd_fbp_forbild.ipynb cells 2-3: 16x16 image, dx=du=0.25, a
    2x2 block of ones, one view at angle 0."""
    p = Proj(nx=16, ny=16, nz=1, dx=0.25, dy=0.25, dz=1, nu=16, nv=1, du=0.25, dv=1, nview=1)
    img = np.zeros([1, 1, 16, 16], np.float32)
    img[0, 0, 7:9, 7:9] = 1
    prj = np.zeros([1, 1, 1, 16], np.float32)
    prj[0, 0, 0, 7:9] = 1
    return "kat", p, dict(img=img, angles=np.zeros(1, np.float32), prj=prj)


def case_siddon():
    p = Proj(nx=48, ny=40, nz=16, dx=1.0, dy=1.0, dz=1.0, nu=64, nv=16, du=1.2858, dv=1.0, nview=24)
    rng = np.random.default_rng(S.seed_for(105))
    feed = 16 * 1.0 * 595.0 / 1085.6
    dc, du, dv, src = S.helical(24, 1.0, 595.0, 1085.6, feed)
    img = np.stack([S.ellipsoid_phantom(rng, 16, 40, 48, 1.0, 1.0, 1.0, supersample=1) for _ in range(2)])
    return "siddon", p, dict(img=img, det_center=dc, det_u=du, det_v=dv, src=src)


def case_tomo():
    p = Proj(nx=48, ny=40, nz=12, dx=1.0, dy=1.0, dz=1.0, nu=64, nv=56, du=1.0, dv=1.0, nview=9)
    rng = np.random.default_rng(S.seed_for(106))
    dc, src = S.tomo_geometry(9, 30.0, 600.0, -20.0)
    img = np.stack([S.ellipsoid_phantom(rng, 12, 40, 48, 1.0, 1.0, 1.0, supersample=1) for _ in range(2)])
    return "tomo", p, dict(img=img, det_center=dc, src=src)


def case_par_wide():
    """Full detector width of the parallel benchmark workload (768 cells of
    0.8 mm) with a coarse image covering it, 24 views."""
    p = Proj(nx=256, ny=256, nz=1, dx=2.4, dy=2.4, nu=768, nv=1, du=0.8, dv=1.0, nview=24)
    rng = np.random.default_rng(S.seed_for(107))
    ang = S.angles(24, np.pi)
    img = _phantom_stack(rng, 1, 1, 256, 256, 2.4, 2.4)
    return "par_wide", p, dict(img=img, angles=ang)


def case_fan_45():
    """Full detector width of the fan workload (736 cells of 1.2858 mm), 24
    views on multiples of 15 degrees -- four of them exactly on 45-degree
    diagonals, where the reference's hard axis switch follows its fast
    intrinsic cos/sin (compared with the reference only)."""
    p = Proj(nx=128, ny=128, nz=1, dx=3.0, dy=3.0, nu=736, nv=1, du=1.2858, dv=1.0, nview=24)
    rng = np.random.default_rng(S.seed_for(108))
    ang = S.angles(24, 2 * np.pi)
    img = _phantom_stack(rng, 1, 1, 128, 128, 3.0, 3.0)
    return "fan_45", p, dict(img=img, angles=ang)


def case_fan_wide():
    """As fan_45 with the views offset by 0.3 degrees (no exact diagonals)."""
    p = Proj(nx=128, ny=128, nz=1, dx=3.0, dy=3.0, nu=736, nv=1, du=1.2858, dv=1.0, nview=24)
    rng = np.random.default_rng(S.seed_for(109))
    ang = (S.angles(24, 2 * np.pi) + np.float32(np.deg2rad(0.3))).astype(np.float32)
    img = _phantom_stack(rng, 1, 1, 128, 128, 3.0, 3.0)
    return "fan_wide", p, dict(img=img, angles=ang)


ALL = [case_fan_basic, case_fan_offsets, case_par_basic, case_par_offsets, case_kat, case_siddon, case_tomo,
       case_par_wide, case_fan_45, case_fan_wide]
