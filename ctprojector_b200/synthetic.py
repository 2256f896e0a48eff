"""Seeded synthetic inputs: ellipse phantoms, Poisson noise and the scan
geometries of the benchmark workloads.

Phantom: a disk of radius R = 0.45 * nx * dx with attenuation 0.019 /mm, plus
ellipses that set the attenuation to U(0.01, 0.03) /mm; centres uniform in a
disk of radius 0.6 R, semi-axes U(0.04, 0.25) R, orientation U(0, pi),
rasterised with super-sampling.  The public phantoms the reference notebooks
use are not available; these stand in for them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def seed_for(config: int, index: int = 0) -> int:
    return 20261203 + 1000 * config + index


def ellipse_phantom(rng: np.random.Generator, nx: int, ny: int, dx: float, dy: float, n_ellipses: int = 10,
                    supersample: int = 4) -> np.ndarray:
    """[ny, nx] float32 phantom in 1/mm (each shape rasterised inside its
    bounding box on the super-sampled grid)."""
    R = 0.45 * nx * dx
    ss = supersample
    xs = ((np.arange(nx * ss) + 0.5) / ss * dx - nx * dx / 2).astype(np.float32)
    ys = ((np.arange(ny * ss) + 0.5) / ss * dy - ny * dy / 2).astype(np.float32)
    img = np.where(xs[None, :] ** 2 + ys[:, None] ** 2 <= R * R, np.float32(0.019), np.float32(0.0))
    for _ in range(n_ellipses):
        r = 0.6 * R * math.sqrt(rng.uniform())
        t = rng.uniform(0, 2 * math.pi)
        x0, y0 = r * math.cos(t), r * math.sin(t)
        a, b = rng.uniform(0.04, 0.25, size=2) * R
        phi = rng.uniform(0, math.pi)
        mu = rng.uniform(0.01, 0.03)
        c, s = math.cos(phi), math.sin(phi)
        ext = max(a, b)
        i0, i1 = np.searchsorted(xs, x0 - ext), np.searchsorted(xs, x0 + ext)
        j0, j1 = np.searchsorted(ys, y0 - ext), np.searchsorted(ys, y0 + ext)
        X = xs[None, i0:i1] - x0
        Y = ys[j0:j1, None] - y0
        u = X * c + Y * s
        v = -X * s + Y * c
        sub = img[j0:j1, i0:i1]
        sub[(u / a) ** 2 + (v / b) ** 2 <= 1] = mu
    img = img.reshape(ny, ss, nx, ss).mean(axis=(1, 3))
    return img.astype(np.float32)


def ellipsoid_phantom(rng: np.random.Generator, nz: int, ny: int, nx: int, dz: float, dy: float, dx: float,
                      n_ellipsoids: int = 10, supersample: int = 2) -> np.ndarray:
    """[nz, ny, nx] float32 phantom: a cylinder plus ellipsoids with z semi-axes
    U(0.1, 0.5) * (nz * dz / 2)."""
    R = 0.45 * nx * dx
    H = nz * dz / 2
    ss = supersample
    xs = (np.arange(nx * ss) + 0.5) / ss * dx - nx * dx / 2
    ys = (np.arange(ny * ss) + 0.5) / ss * dy - ny * dy / 2
    zs = (np.arange(nz) + 0.5) * dz - nz * dz / 2
    X, Y = np.meshgrid(xs, ys)
    base = np.where(X * X + Y * Y <= R * R, 0.019, 0.0)
    ells = []
    for _ in range(n_ellipsoids):
        r = 0.6 * R * math.sqrt(rng.uniform())
        t = rng.uniform(0, 2 * math.pi)
        ells.append(dict(x0=r * math.cos(t), y0=r * math.sin(t), z0=rng.uniform(-0.5, 0.5) * H,
                         a=rng.uniform(0.04, 0.25) * R, b=rng.uniform(0.04, 0.25) * R,
                         c=rng.uniform(0.1, 0.5) * H, phi=rng.uniform(0, math.pi), mu=rng.uniform(0.01, 0.03)))
    out = np.empty((nz, ny, nx), np.float32)
    for k, z in enumerate(zs):
        img = base.copy()
        for e in ells:
            wz = 1 - ((z - e["z0"]) / e["c"]) ** 2
            if wz <= 0:
                continue
            c, s = math.cos(e["phi"]), math.sin(e["phi"])
            u = (X - e["x0"]) * c + (Y - e["y0"]) * s
            v = -(X - e["x0"]) * s + (Y - e["y0"]) * c
            img = np.where((u / e["a"]) ** 2 + (v / e["b"]) ** 2 <= wz, e["mu"], img)
        out[k] = img.reshape(ny, ss, nx, ss).mean(axis=(1, 3))
    return out


def poisson_log(prj: np.ndarray, I0: float, rng: np.random.Generator) -> np.ndarray:
    """-log(counts / I0) with counts ~ Poisson(I0 exp(-p)) clamped to >= 1."""
    counts = rng.poisson(I0 * np.exp(-prj.astype(np.float64)))
    counts = np.maximum(counts, 1)
    return (-np.log(counts / I0)).astype(np.float32)


@dataclass
class Scan:
    """Geometry of one workload (attributes of the reference ct_projector)."""

    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    nu: int
    nv: int
    du: float
    dv: float
    nview: int
    dsd: float = 1085.6
    dso: float = 595.0
    cx: float = 0.0
    cy: float = 0.0
    cz: float = 0.0
    off_u: float = 0.0
    off_v: float = 0.0

    def projector(self, cls):
        p = cls()
        for k, v in self.__dict__.items():
            setattr(p, k, v)
        return p


def angles(nview: int, span: float) -> np.ndarray:
    """nview float32 angles over [0, span), computed like get_angles."""
    return (np.arange(0, nview, dtype=np.float32) * np.float32(span) / np.float32(nview)).astype(np.float32)


def config1() -> tuple[Scan, np.ndarray, int]:
    """Fan-beam FP then BP: 1x1x256x256 at 1 mm, 360 views over 2 pi, 736 cells
    of 1.2858 mm, SID 595, SDD 1085.6."""
    return Scan(256, 256, 1, 1.0, 1.0, 1.0, 736, 1, 1.2858, 1.0, 360), angles(360, 2 * np.pi), 1


def config2() -> tuple[Scan, np.ndarray, int]:
    """Parallel-beam FP/BP + ramp filter FBP: 16 slices 512x512 at 0.8 mm, 720
    views over pi, 768 cells of 0.8 mm."""
    return Scan(512, 512, 1, 0.8, 0.8, 1.0, 768, 1, 0.8, 1.0, 720), angles(720, np.pi), 16


def config4() -> tuple[Scan, np.ndarray, int]:
    """Fan-beam SQS workload: 4x512x512 at 0.8 mm, 984 views over 2 pi, 888
    cells (SID/SDD/cell pitch of config 1, not given for this workload)."""
    return Scan(512, 512, 1, 0.8, 0.8, 1.0, 888, 1, 1.2858, 1.0, 984), angles(984, 2 * np.pi), 4


def helical(nview: int, turns: float, dso: float, dsd: float, feed_per_turn: float, z_center: float = 0.0):
    """Helical cone-beam trajectory: (det_center, det_u, det_v, src), each
    [nview, 3] float32 as (x, y, z).  Source at radius dso; flat detector at
    distance dsd from the source; det_u tangential, det_v along z."""
    th = np.arange(nview, dtype=np.float64) * (2 * np.pi * turns / nview)
    z = z_center + feed_per_turn * (th / (2 * np.pi) - turns / 2)
    c, s = np.cos(th), np.sin(th)
    src = np.stack([dso * c, dso * s, z], axis=1)
    det_center = np.stack([-(dsd - dso) * c, -(dsd - dso) * s, z], axis=1)
    det_u = np.stack([-s, c, np.zeros_like(th)], axis=1)
    det_v = np.tile(np.array([0.0, 0.0, 1.0]), (nview, 1))
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    return f(det_center), f(det_u), f(det_v), f(src)


def config3() -> tuple[Scan, tuple, int]:
    """Helical cone-beam Siddon: 1x64x512x512 at 0.7x0.7x1.0 mm, 1152 views over 2
    turns, pitch 1.0, flat panel 736x64 of 1.2858x1.0 mm, batch 2."""
    scan = Scan(512, 512, 64, 0.7, 0.7, 1.0, 736, 64, 1.2858, 1.0, 1152)
    feed = 1.0 * 64 * 1.0 * scan.dso / scan.dsd
    return scan, helical(1152, 2.0, scan.dso, scan.dsd, feed), 2


def tomo_geometry(nview: int, arc_deg: float, src_height: float, det_z: float):
    """Tomosynthesis: sources on an arc in the x-z plane above a detector plane
    at z = det_z with u = (1,0,0), v = (0,1,0).  Returns (det_center, src)."""
    phi = np.deg2rad(np.linspace(-arc_deg / 2, arc_deg / 2, nview))
    src = np.stack([src_height * np.sin(phi), np.zeros_like(phi), det_z + src_height * np.cos(phi)], axis=1)
    det_center = np.stack([np.zeros_like(phi), np.zeros_like(phi), np.full_like(phi, det_z)], axis=1)
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    return f(det_center), f(src)
