"""Scan protocols and seeded arrival streams of the served reconstruction
workload, as plain data (numpy only: importing this module loads no GPU
library, so a timing run of another implementation can share the stream).

A stream mixes fan-beam (256^2 and 512^2), parallel-beam (512^2) and helical
cone-beam (64 x 512^2) protocols; 2D jobs bring 1-16 slices, cone jobs one
volume.  Each job is an FBP or an SQS-TV reconstruction (SQS for cone).
Arrivals are a Poisson process.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

from .. import synthetic as S

# job-count weights of the mixed stream: equal weight per geometry family,
# split between FBP and SQS-TV for the 2D families
MIX: Dict[str, float] = {
    "fan256_fbp": 1 / 12, "fan256_sqs": 1 / 12, "fan512_fbp": 1 / 12, "fan512_sqs": 1 / 12,
    "par512_fbp": 1 / 6, "par512_sqs": 1 / 6,
    "cone64_sqs": 1 / 3,
}
MIX_2D: Dict[str, float] = {k: v for k, v in MIX.items() if not k.startswith("cone")}


def offset_views(angles: np.ndarray, step: float) -> np.ndarray:
    """Views shifted by half a view step.  No view then lies exactly on a 45
    degree diagonal, where the reference's axis choice (reproduced here with
    the same fast intrinsics) and an exact-trigonometry reconstruction may
    pick different axes for that view."""
    return (angles + np.float32(step / 2)).astype(np.float32)


def protocol_specs(n_iter: int = 20, beta: float = 2e-4, eps: float = 1e-6) -> Dict[str, dict]:
    """Keyword arguments of every protocol of the served stream (name, kind,
    algo, scan, angles or cone geometry, SQS-TV settings); storage types are
    added by the caller.  Views start half a view step past 0; geometry of each
    family: fan 256^2 / 360 views / 736 cells and fan 512^2 / 984 views / 888
    cells at SID 595, SDD 1085.6; parallel 512^2 / 720 views / 768 cells;
    helical cone 64 x 512^2 at 0.7 x 0.7 x 1.0 mm, 360 views over one turn,
    736 x 64 panel."""
    fan256 = S.Scan(256, 256, 1, 1.0, 1.0, 1.0, 736, 1, 1.2858, 1.0, 360)
    fan512 = S.Scan(512, 512, 1, 0.8, 0.8, 1.0, 888, 1, 1.2858, 1.0, 984)
    par512 = S.Scan(512, 512, 1, 0.8, 0.8, 1.0, 768, 1, 0.8, 1.0, 720)
    cone64 = S.Scan(512, 512, 64, 0.7, 0.7, 1.0, 736, 64, 1.2858, 1.0, 360)
    cgeo = S.helical(360, 1.0, cone64.dso, cone64.dsd, 64 * 1.0 * cone64.dso / cone64.dsd)
    full = lambda n: offset_views(S.angles(n, 2 * np.pi), 2 * np.pi / n)  # noqa: E731
    half = lambda n: offset_views(S.angles(n, np.pi), np.pi / n)  # noqa: E731
    sq = dict(n_iter=n_iter, beta=beta, tv_weights=(1.0, 1.0, 1.0), eps=eps)
    spec = {
        "fan256_fbp": dict(kind="fan", algo="fbp", scan=fan256, angles=full(360)),
        "fan256_sqs": dict(kind="fan", algo="sqs", scan=fan256, angles=full(360), **sq),
        "fan512_fbp": dict(kind="fan", algo="fbp", scan=fan512, angles=full(984)),
        "fan512_sqs": dict(kind="fan", algo="sqs", scan=fan512, angles=full(984), **sq),
        "par512_fbp": dict(kind="parallel", algo="fbp", scan=par512, angles=half(720)),
        "par512_sqs": dict(kind="parallel", algo="sqs", scan=par512, angles=half(720), **sq),
        "cone64_sqs": dict(kind="cone", algo="sqs", scan=cone64, cone=cgeo, **sq),
    }
    for name, d in spec.items():
        d["name"] = name
    return spec


def arrivals(n_jobs: int, rate: float, seed: int, mix: Dict[str, float],
             max_slices: int = 16) -> List[Tuple[float, str, int]]:
    """(arrival seconds, protocol name, slices) of a seeded Poisson stream."""
    rng = np.random.default_rng(seed)
    names = sorted(mix)
    w = np.array([mix[k] for k in names], dtype=np.float64)
    w /= w.sum()
    t = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    kinds = rng.choice(len(names), size=n_jobs, p=w)
    nz = rng.integers(1, max_slices + 1, size=n_jobs)
    return [(float(t[i]), names[kinds[i]], int(nz[i])) for i in range(n_jobs)]
