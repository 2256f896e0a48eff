"""FP64 reference reconstructions for the served algorithms (test
infrastructure: the serving tests and the bench check served results against
these; nothing in the product calls them).

Both follow the reference's reconstruction scripts on the oracle's projectors:

* ``fbp``: ramp_filter then the FBP-weighted distance-driven back projection
  (parallel.py / fan_equiangular.py ramp_filter + distance_driven_bp(is_fbp)).
* ``sqs_tv``: n_iter SQS iterations with the TV prior from a zero image,
  x <- x - (A^T (A x - y) + beta s1(x)) / (A^T A 1 + beta s2(x))
  (sqs_one_step, recon/cupy/sqs_algorithms.py:22-57, with weight 1 and the
  projector normalisation folded into beta).

Slices of a 2D job are independent projections (batch of single slices);
the TV prior couples them along z as one volume.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def _proj2d(p):
    class P:
        pass

    q = P()
    for k, v in vars(p).items():
        setattr(q, k, v)
    q.nz = 1
    q.nv = 1
    return q


def _fp(p, kind, x, geo):
    if kind == "cone":
        return O.siddon_fp(p, x, *geo)
    return O.dd_fp(_proj2d(p), x, geo, kind)


def _bp(p, kind, y, geo):
    if kind == "cone":
        return O.siddon_bp(p, y, *geo)
    return O.dd_bp(_proj2d(p), y, geo, kind)


def _layout(p, kind, y):
    """Sinogram of one job -> (batch layout, image shape, zlink of the job)."""
    y = np.asarray(y, dtype=np.float64)
    if kind == "cone":
        nz = int(p.nz)
        img_shape = (1, nz, int(p.ny), int(p.nx))
    else:
        nz = y.shape[0]
        img_shape = (nz, 1, int(p.ny), int(p.nx))
    zl = np.zeros(nz, np.uint8)
    zl[1:] |= 1
    zl[:-1] |= 2
    return y, img_shape, zl


def sqs_tv(p, kind, y, geo, n_iter, beta, weights, eps=1e-8, callback=None):
    """FP64 SQS-TV reconstruction of one job; returns [nz, ny, nx].
    ``callback(k, x)`` (optional) sees every iterate k = 1..n_iter."""
    y, shape, zl = _layout(p, kind, y)
    one = np.ones((1,) + shape[1:])
    norm = _bp(p, kind, _fp(p, kind, one, geo), geo).reshape(-1, shape[-2], shape[-1])
    x = np.zeros(shape)
    for k in range(n_iter):
        r = _fp(p, kind, x, geo) - y
        bp = _bp(p, kind, r, geo)
        x = O.sqs_tv_update(x.reshape(-1, shape[-2], shape[-1]), bp.reshape(-1, shape[-2], shape[-1]), norm, zl,
                            weights, beta, eps).reshape(shape)
        if callback is not None:
            callback(k + 1, x.reshape(-1, shape[-2], shape[-1]))
    return x.reshape(-1, shape[-2], shape[-1])


def fbp(p, kind, y, angles, filter_type="hann"):
    """FP64 FBP of one 2D job (fan or parallel); returns [nz, ny, nx]."""
    q = _proj2d(p)
    f = O.ramp_filter(q, np.asarray(y, dtype=np.float64), filter_type, kind)
    img = O.dd_bp(q, f, angles, kind, is_fbp=True)
    return img.reshape(-1, int(p.ny), int(p.nx))
