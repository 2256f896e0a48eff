"""The plain per-call path: one job at a time, FP32, one public-API call per
operation, as a script written against the reference's cupy modules would do
it (upload the sinogram, compute A^T A 1, run the iterations with
distance_driven_fp / distance_driven_bp or siddon_*_arbitrary, tv_sqs and
array arithmetic, download the image, synchronise).  The server is measured
against this on the same jobs and the same GPU."""
from __future__ import annotations

import time
from collections import deque
from typing import Sequence

import torch

from .. import prior
from ..quant import Q16
from ..projector.cupy import cone as C
from ..projector.cupy import fan_equiangular as F
from ..projector.cupy import parallel as P
from .busy import BusyTracker
from .engine import Job
from .scheduler import LatencyStats


def reconstruct(job: Job) -> torch.Tensor:
    """One job through the public API in FP32; returns the host image [nz, ny, nx]."""
    p = job.protocol
    s = p.scan
    y = job.sinogram.to("cuda").float() if isinstance(job.sinogram, Q16) else job.sinogram.to("cuda", torch.float32)
    if p.kind == "cone":
        geo = [torch.as_tensor(a, device="cuda") for a in p.cone]
        fp = lambda x: C.siddon_fp_arbitrary(s, x, *geo)  # noqa: E731
        bp = lambda r: C.siddon_bp_arbitrary(s, r, *geo)  # noqa: E731
        shape = (1, int(s.nz), int(s.ny), int(s.nx))
    else:
        mod = F if p.kind == "fan" else P
        ang = torch.as_tensor(p.angles, device="cuda")
        if p.algo == "fbp":
            img = mod.distance_driven_bp(s, mod.ramp_filter(s, y, p.filter), ang, True)
            return img.reshape(-1, int(s.ny), int(s.nx)).cpu()
        fp = lambda x: mod.distance_driven_fp(s, x, ang)  # noqa: E731
        bp = lambda r: mod.distance_driven_bp(s, r, ang)  # noqa: E731
        shape = (job.nz, 1, int(s.ny), int(s.nx))
    norm = bp(fp(torch.ones((1,) + shape[1:], device="cuda")))
    x = torch.zeros(shape, device="cuda")
    vol = (1, -1, int(s.ny), int(s.nx))  # the job's slices as one volume for the prior
    for _ in range(p.n_iter):
        g = bp(fp(x) - y)
        s1, s2, _ = prior.tv_sqs(x.reshape(vol), p.tv_weights, p.eps)
        x = x - (g + p.beta * s1.reshape(shape)) / (norm + p.beta * s2.reshape(shape))
    return x.reshape(-1, int(s.ny), int(s.nx)).cpu()


def run_per_call(jobs: Sequence[Job], realtime: bool = True, track_busy: bool = False) -> dict:
    """Serve ``jobs`` one after another in arrival order (each starts when it
    has arrived and the previous one is done).  Fills ``result`` and
    ``t_done``; returns the latency summary (with ``track_busy``, also the
    GPU-busy time of the jobs' work, busy.BusyTracker)."""
    stats = LatencyStats()
    pending = deque(sorted(jobs, key=lambda j: j.arrival))
    tracker = BusyTracker() if track_busy else None
    t0 = time.perf_counter()
    while pending:
        job = pending.popleft()
        if realtime:
            wait = job.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        stream = torch.cuda.current_stream()
        start = tracker.begin(stream) if tracker is not None else None
        job.result = reconstruct(job)
        if start is not None:
            tracker.end(stream, start)
        torch.cuda.synchronize()
        job.t_done = time.perf_counter() - t0
        stats.add(job.latency, job.t_done)
    wall = time.perf_counter() - t0
    summary = stats.summary(0.0)
    if tracker is not None:
        busy = tracker.busy_seconds()
        summary.update(wall_s=wall, gpu_busy_s=busy, gpu_busy_frac=busy / wall if wall > 0 else 0.0)
    return summary
