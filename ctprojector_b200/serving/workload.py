"""Seeded synthetic job streams for the reconstruction server: the protocols
and arrivals of ``mix`` as engine Protocols and Jobs.  Sinograms are seeded
ellipse / ellipsoid phantoms projected with the FP32 projectors, with Poisson noise at the given
photon count before the -log transform, drawn from a small pool per protocol
(the content of a job does not change its cost).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import quant
from .. import synthetic as S
from ..projector import _device as D
from .engine import DTYPES, Job, Protocol
from .mix import MIX, MIX_2D, arrivals, protocol_specs  # noqa: F401  (re-exported)


def catalog(storage: str = "bfloat16", n_iter: int = 20, image_storage: str = "float32",
            beta: float = 2e-4, eps: float = 1e-6) -> Dict[str, Protocol]:
    """The protocols of the served stream (``mix.protocol_specs``) with the
    sinogram storage type ``storage`` and, for SQS protocols, the iterate
    storage type ``image_storage``."""
    out = {}
    for name, d in protocol_specs(n_iter=n_iter, beta=beta, eps=eps).items():
        kw = dict(d, storage=storage)
        if d["algo"] == "sqs":
            kw["image_storage"] = image_storage
        out[name] = Protocol(**kw)
    return out


def sinogram_pool(p: Protocol, n_variants: int, max_slices: int, seed: int, photons: float = 1e5) -> List[torch.Tensor]:
    """Pinned host sinograms of ``p`` (``max_slices`` slices for 2D, one volume
    for cone) in the protocol's storage type (a ``quant.Q16`` for q16)."""
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
        if p.storage == "q16":  # quantized on the device, kept in pinned host memory
            out.append(quant.quantize(y.cuda()).cpu().pin_memory())
        else:
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
