"""Seeded synthetic job streams for the reconstruction server.

A stream mixes fan-beam (256^2 and 512^2), parallel-beam (512^2) and helical
cone-beam (64 x 512^2) protocols; 2D jobs bring 1-16 slices, cone jobs one
volume.  Each job is an FBP or an SQS-TV reconstruction (SQS for cone).
Arrivals are a Poisson process.  Sinograms are seeded ellipse / ellipsoid
phantoms projected with the FP32 projectors, with Poisson noise at the given
photon count before the -log transform, drawn from a small pool per protocol
(the content of a job does not change its cost).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import synthetic as S
from ..projector import _device as D
from .engine import DTYPES, Job, Protocol

# job-count weights of the mixed stream: equal weight per geometry family,
# split between FBP and SQS-TV for the 2D families
MIX: Dict[str, float] = {
    "fan256_fbp": 1 / 12, "fan256_sqs": 1 / 12, "fan512_fbp": 1 / 12, "fan512_sqs": 1 / 12,
    "par512_fbp": 1 / 6, "par512_sqs": 1 / 6,
    "cone64_sqs": 1 / 3,
}
MIX_2D: Dict[str, float] = {k: v for k, v in MIX.items() if not k.startswith("cone")}


def _offset(angles: np.ndarray, step: float) -> np.ndarray:
    """Views shifted by half a view step.  No view then lies exactly on a 45
    degree diagonal, where the reference's axis choice (reproduced here with
    the same fast intrinsics) and an exact-trigonometry reconstruction may
    pick different axes for that view."""
    return (angles + np.float32(step / 2)).astype(np.float32)


def catalog(storage: str = "bfloat16", n_iter: int = 20, image_storage: str = "float32",
            beta: float = 2e-4, eps: float = 1e-6) -> Dict[str, Protocol]:
    """The protocols of the served stream (views start half a view step past
    0; geometry of each family as in the projector workloads: fan 256^2 / 360 views / 736 cells and fan 512^2 / 984
    views / 888 cells at SID 595, SDD 1085.6; parallel 512^2 / 720 views / 768
    cells; helical cone 64 x 512^2 at 0.7 x 0.7 x 1.0 mm, 360 views over one
    turn, 736 x 64 panel)."""
    fan256 = S.Scan(256, 256, 1, 1.0, 1.0, 1.0, 736, 1, 1.2858, 1.0, 360)
    fan512 = S.Scan(512, 512, 1, 0.8, 0.8, 1.0, 888, 1, 1.2858, 1.0, 984)
    par512 = S.Scan(512, 512, 1, 0.8, 0.8, 1.0, 768, 1, 0.8, 1.0, 720)
    cone64 = S.Scan(512, 512, 64, 0.7, 0.7, 1.0, 736, 64, 1.2858, 1.0, 360)
    cgeo = S.helical(360, 1.0, cone64.dso, cone64.dsd, 64 * 1.0 * cone64.dso / cone64.dsd)
    full = lambda n: _offset(S.angles(n, 2 * np.pi), 2 * np.pi / n)  # noqa: E731
    half = lambda n: _offset(S.angles(n, np.pi), np.pi / n)  # noqa: E731
    sq = dict(n_iter=n_iter, beta=beta, tv_weights=(1.0, 1.0, 1.0), eps=eps, storage=storage,
              image_storage=image_storage)
    return {
        "fan256_fbp": Protocol("fan256_fbp", "fan", "fbp", fan256, angles=full(360), storage=storage),
        "fan256_sqs": Protocol("fan256_sqs", "fan", "sqs", fan256, angles=full(360), **sq),
        "fan512_fbp": Protocol("fan512_fbp", "fan", "fbp", fan512, angles=full(984), storage=storage),
        "fan512_sqs": Protocol("fan512_sqs", "fan", "sqs", fan512, angles=full(984), **sq),
        "par512_fbp": Protocol("par512_fbp", "parallel", "fbp", par512, angles=half(720), storage=storage),
        "par512_sqs": Protocol("par512_sqs", "parallel", "sqs", par512, angles=half(720), **sq),
        "cone64_sqs": Protocol("cone64_sqs", "cone", "sqs", cone64, cone=cgeo, **sq),
    }


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


def sinogram_pool(p: Protocol, n_variants: int, max_slices: int, seed: int, photons: float = 1e5) -> List[torch.Tensor]:
    """Pinned host sinograms of ``p`` (``max_slices`` slices for 2D, one volume
    for cone) in the protocol's storage type."""
    rng = np.random.default_rng(seed)
    s = p.scan
    out = []
    for _ in range(n_variants):
        if p.kind == "cone":
            vol = S.ellipsoid_phantom(rng, int(s.nz), int(s.ny), int(s.nx), s.dz, s.dy, s.dx, supersample=1)[None]
            geo = [torch.tensor(a, device="cuda") for a in p.cone]
            y = D.siddon_fp(s, torch.tensor(vol, device="cuda"), *geo)
        else:
            img = np.stack([S.ellipse_phantom(rng, int(s.nx), int(s.ny), s.dx, s.dy)[None]
                            for _ in range(max_slices)])
            geom = 0 if p.kind == "fan" else 1
            y = D.dd_fp(s, torch.tensor(img, device="cuda"), torch.tensor(p.angles, device="cuda"), geom)
        y = torch.tensor(S.poisson_log(y.cpu().numpy(), photons, rng))
        out.append(y.to(DTYPES[p.storage]).pin_memory())
    return out


def make_jobs(protocols: Dict[str, Protocol], stream: Sequence[Tuple[float, str, int]],
              pools: Optional[Dict[str, List[torch.Tensor]]] = None, seed: int = 0,
              max_slices: int = 16) -> List[Job]:
    """Jobs of ``stream``; sinograms are views into per-protocol pools (built
    here when not given)."""
    rng = np.random.default_rng(seed)
    if pools is None:
        pools = {name: sinogram_pool(protocols[name], 2, max_slices, seed + i)
                 for i, name in enumerate(sorted({n for _, n, _ in stream}))}
    jobs = []
    for i, (t, name, nz) in enumerate(stream):
        p = protocols[name]
        k = int(rng.integers(len(pools[name])))
        src = pools[name][k]
        if p.kind == "cone":
            nz, sino = int(p.scan.nz), src
        else:
            sino = src[:nz]
        jobs.append(Job(i, p, sino, arrival=t, nz=nz, tag=(name, k)))
    return jobs


def same_jobs(jobs: Sequence[Job], protocols: Dict[str, Protocol], pools: Dict[str, List[torch.Tensor]]) -> List[Job]:
    """The jobs of ``jobs`` (same arrivals, slices and data source) on other
    protocols and pools, e.g. the float32 versions for the per-call path."""
    out = []
    for j in jobs:
        name, k = j.tag
        src = pools[name][k]
        sino = src if j.protocol.kind == "cone" else src[:j.nz]
        out.append(Job(j.job_id, protocols[name], sino, arrival=j.arrival, nz=j.nz, tag=j.tag))
    return out
