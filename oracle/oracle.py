"""CPU FP64 oracle for the CTProjector projector pair.

TEST INFRASTRUCTURE ONLY.  The parity tests, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` leg of ``bench.py`` use this module to check results and
to time the CPU baseline; the ``ctprojector_b200`` product never imports it.

The distance-driven, Siddon, tomosynthesis and ``fbp_bp`` operators are the C
restatement in ``ctp_oracle.c`` (FP64, OpenMP).  The ramp filter is restated
here in numpy float64, following ``fbpMath.cu:90-267`` (``GetRamp``),
``fbpParallel.cu:14-109`` and ``fbp.cu:15-162`` of the reference
(src/ct_projector/kernel/projector/cuda/).

Every function takes the same ``projector`` object the reference Python
wrappers take (attributes nx, ny, nz, dx, ..., du, dv, off_u, off_v, dsd, dso)
and follows the argument conventions of the reference wrapper it names.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, Structure, c_double, c_float, c_int, c_long, c_longlong

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_SRC_PATH = os.path.join(_HERE, "ctp_oracle.c")


def build(force: bool = False) -> str:
    """Compile ctp_oracle.c into liboracle.so next to it (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(_SRC_PATH):
        cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11", _SRC_PATH, "-o", _LIB_PATH, "-lm"]
        subprocess.run(cmd, check=True)
    return _LIB_PATH


class _Grid(Structure):
    _fields_ = [("nx", c_long), ("ny", c_long), ("nz", c_long),
                ("dx", c_double), ("dy", c_double), ("dz", c_double),
                ("cx", c_double), ("cy", c_double), ("cz", c_double)]


class _Det(Structure):
    _fields_ = [("nu", c_long), ("nv", c_long),
                ("du", c_double), ("dv", c_double), ("off_u", c_double), ("off_v", c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = POINTER(c_double)
        fp = POINTER(c_float)
        L.oracle_dd2d_fp.argtypes = [dp, dp, dp, c_long, _Grid, _Det, c_long, c_double, c_double, c_int]
        L.oracle_dd2d_fp_mode.argtypes = [dp, dp, dp, c_long, _Grid, _Det, c_long, c_double, c_double, c_int, c_int]
        L.oracle_dd2d_bp_adjoint.argtypes = [dp, dp, dp, c_long, _Grid, _Det, c_long, c_double, c_double, c_int]
        L.oracle_dd2d_nnz.argtypes = [dp, _Grid, _Det, c_long, c_double, c_double, c_int]
        L.oracle_dd2d_nnz.restype = c_longlong
        L.oracle_dd2d_bp.argtypes = [dp, dp, dp, c_long, _Grid, _Det, c_long, c_double, c_double, c_int, c_int]
        L.oracle_dd2d_bp_mode.argtypes = [dp, dp, dp, c_long, _Grid, _Det, c_long, c_double, c_double, c_int, c_int,
                                          c_int]
        L.oracle_fbp_fan_bp.argtypes = [dp, dp, dp, c_long, _Grid, _Det, c_long, c_double, c_double]
        L.oracle_siddon_fp.argtypes = [dp, dp, fp, fp, fp, fp, c_long, _Grid, _Det, c_long]
        L.oracle_siddon_bp.argtypes = [dp, dp, fp, fp, fp, fp, c_long, _Grid, _Det, c_long]
        L.oracle_siddon_nnz.argtypes = [fp, fp, fp, fp, _Grid, _Det, c_long]
        L.oracle_siddon_fan_fp.argtypes = [dp, dp, dp, c_long, _Grid, _Det, c_long, c_double, c_double]
        L.oracle_siddon_fan_bp.argtypes = [dp, dp, dp, c_long, _Grid, _Det, c_long, c_double, c_double]
        L.oracle_siddon_nnz.restype = c_longlong
        L.oracle_tomo_fp.argtypes = [dp, dp, fp, fp, c_long, _Grid, _Det, c_long]
        L.oracle_tomo_bp.argtypes = [dp, dp, fp, fp, c_long, _Grid, _Det, c_long]
        L.oracle_num_threads.restype = c_int
        _lib = L
    return _lib


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def _grid(p, shape=None):
    nz, ny, nx = (shape if shape is not None else (p.nz, p.ny, p.nx))
    return _Grid(int(nx), int(ny), int(nz), float(np.float32(p.dx)), float(np.float32(p.dy)),
                 float(np.float32(p.dz)), float(np.float32(p.cx)), float(np.float32(p.cy)),
                 float(np.float32(p.cz)))


def _det(p, nu, nv, du=None):
    du = p.du if du is None else du
    return _Det(int(nu), int(nv), float(np.float32(du)), float(np.float32(p.dv)),
                float(np.float32(p.off_u)), float(np.float32(p.off_v)))


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f3(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a, t=c_double):
    return a.ctypes.data_as(POINTER(t))


def _fan_da(p):
    # The reference wrappers pass c_float(projector.du / projector.dsd).
    return float(np.float32(p.du / p.dsd))


# --------------------------------------------------------------------------- DD 2D
def dd_fp(p, img, angles, geom: str, branchless=False):
    """Fan (geom='fan') or parallel DD forward projection.  Mirrors
    fan_equiangular.distance_driven_fp / parallel.distance_driven_fp;
    branchless=True traces like the reference's branchless mode (the main
    axis alone, no blend band)."""
    img = _d(img)
    ang = _d(angles)
    nb = img.shape[0]
    prj = np.zeros([nb, len(ang), int(p.nv), int(p.nu)], np.float64)
    g = _grid(p, img.shape[1:])
    if geom == "fan":
        d = _det(p, p.nu, p.nv, _fan_da(p))
        lib().oracle_dd2d_fp_mode(_ptr(prj), _ptr(img), _ptr(ang), nb, g, d, len(ang), float(np.float32(p.dsd)),
                                  float(np.float32(p.dso)), 0, int(bool(branchless)))
    else:
        d = _det(p, p.nu, p.nv)
        lib().oracle_dd2d_fp_mode(_ptr(prj), _ptr(img), _ptr(ang), nb, g, d, len(ang), 1000.0, 500.0, 1,
                                  int(bool(branchless)))
    return prj


def dd_bp(p, prj, angles, geom: str, is_fbp=False, adjoint=False, branchless=False):
    """DD back projection: reference-parity normalised mode, FBP mode, or the
    exact transpose of dd_fp (adjoint=True); branchless=True as the
    reference's branchless mode (parallel: no blend band; detector rows
    interpolated at the pixel's v)."""
    prj = _d(prj)
    ang = _d(angles)
    nb, nview, nv, nu = prj.shape
    img = np.zeros([nb, int(p.nz), int(p.ny), int(p.nx)], np.float64)
    g = _grid(p)
    if geom == "fan":
        d = _det(p, nu, nv, _fan_da(p))
        dsd, dso, gi = float(np.float32(p.dsd)), float(np.float32(p.dso)), 0
    else:
        d = _det(p, nu, nv)
        dsd, dso, gi = 1000.0, 500.0, 1
    if adjoint:
        lib().oracle_dd2d_bp_adjoint(_ptr(img), _ptr(prj), _ptr(ang), nb, g, d, nview, dsd, dso, gi)
    else:
        lib().oracle_dd2d_bp_mode(_ptr(img), _ptr(prj), _ptr(ang), nb, g, d, nview, dsd, dso, gi, int(bool(is_fbp)),
                                  int(bool(branchless)))
    return img


def dd_nnz(p, angles, geom: str, shape=None) -> int:
    ang = _d(angles)
    g = _grid(p, shape)
    if geom == "fan":
        return int(lib().oracle_dd2d_nnz(_ptr(ang), g, _det(p, p.nu, p.nv, _fan_da(p)), len(ang),
                                         float(np.float32(p.dsd)), float(np.float32(p.dso)), 0))
    return int(lib().oracle_dd2d_nnz(_ptr(ang), g, _det(p, p.nu, p.nv), len(ang), 1000.0, 500.0, 1))


def fbp_bp(p, prj, angles):
    """Pixel-driven fan FBP back projection (fan_equiangular.fbp_bp)."""
    prj = _d(prj)
    ang = _d(angles)
    nb, nview, nv, nu = prj.shape
    img = np.zeros([nb, int(p.nz), int(p.ny), int(p.nx)], np.float64)
    lib().oracle_fbp_fan_bp(_ptr(img), _ptr(prj), _ptr(ang), nb, _grid(p), _det(p, nu, nv, _fan_da(p)), nview,
                            float(np.float32(p.dsd)), float(np.float32(p.dso)))
    return img


# --------------------------------------------------------------------------- Siddon cone
def siddon_fp(p, img, det_center, det_u, det_v, src):
    """cone.siddon_fp_arbitrary: geometry arrays [nview, 3] as (x, y, z)."""
    img = _d(img)
    dc, du_, dv_, sr = _f3(det_center), _f3(det_u), _f3(det_v), _f3(src)
    nb = img.shape[0]
    nview = dc.shape[0]
    prj = np.zeros([nb, nview, int(p.nv), int(p.nu)], np.float64)
    lib().oracle_siddon_fp(_ptr(prj), _ptr(img), _ptr(dc, c_float), _ptr(du_, c_float), _ptr(dv_, c_float),
                           _ptr(sr, c_float), nb, _grid(p, img.shape[1:]), _det(p, p.nu, p.nv), nview)
    return prj


def siddon_bp(p, prj, det_center, det_u, det_v, src):
    prj = _d(prj)
    dc, du_, dv_, sr = _f3(det_center), _f3(det_u), _f3(det_v), _f3(src)
    nb, nview, nv, nu = prj.shape
    img = np.zeros([nb, int(p.nz), int(p.ny), int(p.nx)], np.float64)
    lib().oracle_siddon_bp(_ptr(img), _ptr(prj), _ptr(dc, c_float), _ptr(du_, c_float), _ptr(dv_, c_float),
                           _ptr(sr, c_float), nb, _grid(p), _det(p, nu, nv), nview)
    return img


def siddon_nnz(p, det_center, det_u, det_v, src, shape=None) -> int:
    dc, du_, dv_, sr = _f3(det_center), _f3(det_u), _f3(det_v), _f3(src)
    return int(lib().oracle_siddon_nnz(_ptr(dc, c_float), _ptr(du_, c_float), _ptr(dv_, c_float),
                                       _ptr(sr, c_float), _grid(p, shape), _det(p, p.nu, p.nv), dc.shape[0]))


# --------------------------------------------------------------------------- tomo
def tomo_fp(p, img, det_center, src):
    img = _d(img)
    dc, sr = _f3(det_center), _f3(src)
    nb = img.shape[0]
    prj = np.zeros([nb, dc.shape[0], int(p.nv), int(p.nu)], np.float64)
    lib().oracle_tomo_fp(_ptr(prj), _ptr(img), _ptr(dc, c_float), _ptr(sr, c_float), nb, _grid(p, img.shape[1:]),
                         _det(p, p.nu, p.nv), dc.shape[0])
    return prj


def tomo_bp(p, prj, det_center, src):
    prj = _d(prj)
    dc, sr = _f3(det_center), _f3(src)
    nb, nview, nv, nu = prj.shape
    img = np.zeros([nb, int(p.nz), int(p.ny), int(p.nx)], np.float64)
    lib().oracle_tomo_bp(_ptr(img), _ptr(prj), _ptr(dc, c_float), _ptr(sr, c_float), nb, _grid(p),
                         _det(p, nu, nv), nview)
    return img


# --------------------------------------------------------------------------- ramp filter
FILTERS = {"hamming": 1, "hann": 2, "cosine": 3}


def filter_code(filter_type: str) -> int:
    """fan_equiangular.ramp_filter / parallel.ramp_filter: unknown names are RL (0)."""
    return FILTERS.get(filter_type.lower(), 0)


def ramp_kernel(nu: int, da: float, ifilter: int, equiangular: bool) -> np.ndarray:
    """Windowed spatial ramp of length 2nu-1, index i <-> offset i-(nu-1).

    GetRamp, fbpMath.cu:90-241: spatial ramp, FFT, window, inverse FFT, real
    part divided by the length."""
    L = 2 * nu - 1
    k = np.arange(L) - (nu - 1)
    h = np.zeros(L)
    h[k == 0] = 1.0 / (4 * da * da)
    odd = (k % 2) != 0
    if equiangular:
        h[odd] = -1.0 / (np.pi ** 2 * np.sin(k[odd] * da) ** 2)
    else:
        h[odd] = -1.0 / (np.pi ** 2 * k[odd].astype(np.float64) ** 2 * da * da)
    i = np.arange(L)
    if ifilter == 1:
        w = 0.54 + 0.46 * np.cos(2 * np.pi * i / L)
    elif ifilter == 2:
        w = 0.5 + 0.5 * np.cos(2 * np.pi * i / L)
    elif ifilter == 3:
        w = np.abs(np.cos(np.pi * i / L))
    else:
        w = np.ones(L)
    return np.real(np.fft.ifft(np.fft.fft(h) * w))


def ramp_filter(p, prj, filter_type: str = "hann", geom: str = "parallel"):
    """parallel.ramp_filter / fan_equiangular.ramp_filter.

    Each detector row is zero padded, convolved with the windowed ramp and
    cropped: out[i] = scale * sum_j p[j] g[i - j + nu - 1]
    (fbpParallel.cu:56-86, fbp.cu:50-134).  Fan rows are pre-weighted by
    cos(((i - (nu-1)/2) - off_u) da) (fbp.cu:60-67)."""
    prj = _d(prj)
    nb, nview, nv, nu = prj.shape
    ifilter = filter_code(filter_type)
    if geom == "fan":
        da = _fan_da(p)
        g = ramp_kernel(nu, da, ifilter, equiangular=True)
        wgt = np.cos(((np.arange(nu) - (nu - 1) / 2.0) - float(np.float32(p.off_u))) * da)
        x = prj * wgt
        scale = np.pi / nview * da / float(np.float32(p.dso))
    else:
        du = float(np.float32(p.du))
        g = ramp_kernel(nu, du, ifilter, equiangular=False)
        x = prj
        scale = np.pi / nview * du
    n = 1
    while n < 3 * nu - 2:
        n *= 2
    X = np.fft.rfft(x, n=n, axis=-1)
    G = np.fft.rfft(g, n=n)
    full = np.fft.irfft(X * G, n=n, axis=-1)
    return full[..., nu - 1: 2 * nu - 1] * scale


# --------------------------------------------------------------------------- TV prior
def tv_sqs(img, weights, eps=1e-8):
    """SQS terms of the anisotropic TV prior, kernel/prior/cuda/TotalVariation.cu:21-149
    of the reference.  weights along (z, y, x); img [batch, nz, ny, nx]."""
    x = _d(img)
    wz, wy, wx = (float(np.float32(w)) for w in weights)
    dx = np.zeros_like(x)
    dy = np.zeros_like(x)
    dz = np.zeros_like(x)
    dx[..., 1:] = x[..., 1:] - x[..., :-1]
    dy[..., 1:, :] = x[..., 1:, :] - x[..., :-1, :]
    dz[..., 1:, :, :] = x[..., 1:, :, :] - x[..., :-1, :, :]
    var = np.sqrt(wx * dx * dx + wy * dy * dy + wz * dz * dz + float(np.float32(eps)))
    dx1 = np.zeros_like(x)
    dy1 = np.zeros_like(x)
    dz1 = np.zeros_like(x)
    dx1[..., :-1] = x[..., :-1] - x[..., 1:]
    dy1[..., :-1, :] = x[..., :-1, :] - x[..., 1:, :]
    dz1[..., :-1, :, :] = x[..., :-1, :, :] - x[..., 1:, :, :]
    varx = var.copy()
    vary = var.copy()
    varz = var.copy()
    varx[..., :-1] = var[..., 1:]
    vary[..., :-1, :] = var[..., 1:, :]
    varz[..., :-1, :, :] = var[..., 1:, :, :]
    s1 = (wx * dx + wy * dy + wz * dz) / var + wx * dx1 / varx + wy * dy1 / vary + wz * dz1 / varz
    s2 = (wx + wy + wz) / var + wx / varx + wy / vary + wz / varz
    return s1, s2, var


def split_volumes(zlink):
    """Slice ranges [a, b) of the volumes packed in a flat slice array, from the
    per-slice z links (bit 0: neighbour below in the same volume, bit 1: above)."""
    zl = np.asarray(zlink, dtype=np.uint8)
    out, a = [], 0
    for i in range(len(zl)):
        if not (zl[i] & 2):
            out.append((a, i + 1))
            a = i + 1
    return out


def sqs_tv_update(x, bp, norm, zlink, weights, beta, eps=1e-8):
    """x - (bp + beta s1(x)) / (norm + beta s2(x)) in FP64 on a flat slice array
    [nslices, ny, nx]: one SQS iteration with the TV prior (sqs_one_step,
    recon/cupy/sqs_algorithms.py:22-57 of the reference), TV terms per packed
    volume as in tv_sqs.  norm has norm_slices slices, read at i % norm_slices."""
    x = _d(x)
    n = x.shape[0]
    norm = _d(norm)
    idx = np.arange(n) % norm.shape[0]
    s1 = np.zeros_like(x)
    s2 = np.zeros_like(x)
    vols = split_volumes(zlink) if zlink is not None else [(i, i + 1) for i in range(n)]
    for a, b in vols:
        t1, t2, _ = tv_sqs(x[None, a:b], weights, eps)
        s1[a:b], s2[a:b] = t1[0], t2[0]
    beta = float(np.float32(beta))
    return x - (_d(bp) + beta * s1) / (norm[idx] + beta * s2)


def tomo_filter(p, prj, det_center, src, filter_type="hann", cutoff_x=1.0, cutoff_z=1.0, first_view_kernel=False):
    """Tomosynthesis FBP filter in FP64 (fbpTomo::Filter and GetRampTomo,
    kernel/projector/cuda/fbpTomo.cu:50-384 of the reference).  Per view: the
    tilt from the source-to-detector-centre direction in the x-z plane
    (:127-135), the ramp at the virtual pitch vdu = du cos(tilt), windowed in
    frequency by (x window) * (z window) whose frequencies are
    fu * cos * dx * 2 and fu * sin * dz * 2, each clamped above at its cut-off
    (GetFrequency :50-68); every row of the view is convolved with it and
    scaled by pi / nview * vdu (:311, with the transforms' 1/L).

    ``first_view_kernel`` reproduces what the reference computes: it builds
    every view's kernel but multiplies each view's spectrum by the first one
    (FilterByFreqMultiply1D is given pcuFilter without a view offset,
    fbpTomo.cu:323), keeping each view's own scale."""
    prj = _d(prj)
    dc, sr = _d(det_center), _d(src)
    nb, nview, nv, nu = prj.shape
    L = 2 * nu - 1
    du, dx, dz = (float(np.float32(v)) for v in (p.du, p.dx, p.dz))
    cx, cz = float(np.float32(cutoff_x)), float(np.float32(cutoff_z))
    ft = filter_type.lower()
    ifilter = 1 if ft == "hamming" else 2 if ft == "hann" else 0
    k = np.arange(L) - (nu - 1)
    i = np.arange(L)
    n = 1
    while n < 3 * nu - 2:
        n *= 2
    out = np.zeros_like(prj)
    for v in range(nview):
        ddx, ddz = dc[v, 0] - sr[v, 0], dc[v, 2] - sr[v, 2]
        r = np.sqrt(ddx * ddx + ddz * ddz)
        sin_t, cos_t = ddx / r, -ddz / r
        scale_vdu = du * cos_t
        if first_view_kernel:
            ddx, ddz = dc[0, 0] - sr[0, 0], dc[0, 2] - sr[0, 2]
            r = np.sqrt(ddx * ddx + ddz * ddz)
            sin_t, cos_t = ddx / r, -ddz / r
        vdu = du * cos_t
        h = np.zeros(L)
        h[k == 0] = 1.0 / (4 * vdu * vdu)
        odd = (k % 2) != 0
        h[odd] = -1.0 / (np.pi ** 2 * k[odd].astype(np.float64) ** 2 * vdu * vdu)
        fu = np.where(i > (L + 1) // 2, (i - L) / L / vdu, i / L / vdu)
        wx = np.minimum(fu * cos_t * dx * 2, cx)
        wz = np.minimum(fu * sin_t * dz * 2, cz)
        if ifilter == 1:
            w = (0.54 + 0.46 * np.cos(np.pi * wx / cx)) * (0.54 + 0.46 * np.cos(np.pi * wz / cz))
        elif ifilter == 2:
            w = (0.5 + 0.5 * np.cos(np.pi * wx / cx)) * (0.5 + 0.5 * np.cos(np.pi * wz / cz))
        else:
            w = np.ones(L)
        g = np.real(np.fft.ifft(np.fft.fft(h) * w))
        X = np.fft.rfft(prj[:, v], n=n, axis=-1)
        full = np.fft.irfft(X * np.fft.rfft(g, n=n), n=n, axis=-1)
        out[:, v] = full[..., nu - 1: 2 * nu - 1] * (np.pi / nview * scale_vdu)
    return out


def siddon_fan_fp(p, img, angles):
    """fan_equiangluar.siddon_fp (numpy module): fan-beam Siddon rays,
    siddonFan.cu:12-44 (angular cell size du / dsd)."""
    img = _d(img)
    ang = _d(angles)
    nb = img.shape[0]
    prj = np.zeros([nb, len(ang), int(p.nv), int(p.nu)], np.float64)
    lib().oracle_siddon_fan_fp(_ptr(prj), _ptr(img), _ptr(ang), nb, _grid(p, img.shape[1:]),
                               _det(p, p.nu, p.nv, _fan_da(p)), len(ang), float(np.float32(p.dsd)),
                               float(np.float32(p.dso)))
    return prj


def siddon_fan_bp(p, prj, angles):
    """fan_equiangluar.siddon_bp: the transpose of siddon_fan_fp."""
    prj = _d(prj)
    ang = _d(angles)
    nb, nview, nv, nu = prj.shape
    img = np.zeros([nb, int(p.nz), int(p.ny), int(p.nx)], np.float64)
    lib().oracle_siddon_fan_bp(_ptr(img), _ptr(prj), _ptr(ang), nb, _grid(p), _det(p, nu, nv, _fan_da(p)), nview,
                               float(np.float32(p.dsd)), float(np.float32(p.dso)))
    return img


def pixel_bp_parallel(p, prj, angles):
    """parallel.pixel_driven_bp (numpy module; bpParallelKernel3D,
    fbpParallel.cu:200-250): per pixel centre and view the detector position
    pu = -((x cos + y sin)/du + off_u) + (nu-1)/2, pv per slice, bilinear
    interpolation that returns 0 outside [0, n) (InterpolateXY with truncate,
    cudaMath.cu:227-260), summed over views without weights."""
    prj = _d(prj)
    ang = _d(angles)
    nb, nview, nv, nu = prj.shape
    nx, ny, nz = int(p.nx), int(p.ny), int(p.nz)
    f = lambda v: float(np.float32(v))  # noqa: E731
    dx, dy, dz, cx, cy, cz = (f(getattr(p, k)) for k in ("dx", "dy", "dz", "cx", "cy", "cz"))
    du, dv, off_u, off_v = f(p.du), f(p.dv), f(p.off_u), f(p.off_v)
    x = (np.arange(nx) + 0.5 - nx / 2.0) * dx + cx
    y = (np.arange(ny) + 0.5 - ny / 2.0) * dy + cy
    z = (np.arange(nz) + 0.5 - nz / 2.0) * dz + cz
    X, Y = np.meshgrid(x, y)
    img = np.zeros([nb, nz, ny, nx])
    pv = z / dv + off_v + (nv - 1) / 2.0
    for v in range(nview):
        c, s = np.cos(ang[v]), np.sin(ang[v])
        pu = -((X * c + Y * s) / du + off_u) + (nu - 1) / 2.0
        uin = (pu >= 0) & (pu < nu)
        i0 = np.clip(np.floor(pu).astype(np.int64), 0, nu - 1)
        i1 = np.clip(i0 + 1, 0, nu - 1)
        wu = np.where(uin, pu - i0, 0.0)
        for iz in range(nz):
            if not (0 <= pv[iz] < nv):
                continue
            j0 = int(np.floor(pv[iz]))
            j1 = min(j0 + 1, nv - 1)
            wv = pv[iz] - j0
            r0, r1 = prj[:, v, j0], prj[:, v, j1]
            val = (r0[:, i0] * (1 - wu) * (1 - wv) + r0[:, i1] * wu * (1 - wv) + r1[:, i0] * (1 - wu) * wv +
                   r1[:, i1] * wu * wv)
            img[:, iz] += np.where(uin, val, 0.0)
    return img

