"""Continuous-batching reconstruction server on one GPU.

Jobs (an FBP or an SQS-TV reconstruction of one scan) arrive over time.  Jobs
whose scan protocol (geometry + algorithm) is the same share a *lane*: one set
of device-resident buffers with a fixed number of slots (image slices for the
fan/parallel protocols, volumes for cone) and captured CUDA graphs; the
lanes enqueue on the engine's stream (or one stream each, ``lane_streams``).
Each pass of the server loop

1. moves arrived jobs to the arrival queue,
2. admits queued jobs into free slots (creating a lane if the HBM budget
   allows it, after tearing down idle lanes), uploading their sinograms on the
   lane's stream,
3. advances every lane with work by one step (one SQS iteration over all its
   live slots, or one batched FBP), unless its previous-but-one step is still
   running, so the lanes' steps interleave on the GPU and stay at most two
   steps ahead of the host,
4. retires finished jobs: a device-to-host copy of their slots into pinned
   memory, then the slots are freed and the live ones packed to the front.

So a job that arrives while others are on the GPU joins its lane at the next
iteration boundary instead of waiting for the batch to drain.  Slots of one
lane are independent in every kernel (projections are per slice or per
volume; the TV prior stops at each job's own z borders through the per-slice
z links), so a job's result does not depend on what else is in the lane.

The SQS iteration is the reference's sqs_one_step with the TV prior
(recon/cupy/sqs_algorithms.py:22-57, prior/cupy/recon_prior.py:85-135), with
weight 1, x0 = 0 and the projector normalisation folded into beta:

    x <- x - (A^T (A x - y) + beta s1(x)) / (A^T A 1 + beta s2(x))

Storage precision: the measured sinogram is held on the device in the job's
storage type (float32, bfloat16, float16, or "q16": 16-bit codes with one FP32
offset and step per view, ``ctprojector_b200.quant``); the iterate, the
projections of each iteration and every sum are float32.  Optionally the forward projector
reads a low-precision copy of the iterate written by the fused update
(``image_storage``).
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _lib
from .. import quant
from ..projector import _device as D
from ..recon import sqs_tv_update
from .busy import BusyTracker
from .scheduler import ArrivalQueue, LatencyStats, MemoryBudget, Pending, SlotPool, bucket, bucket_sizes

# storage name -> device dtype of the sinogram buffer ("q16": the codes of
# 16-bit affine storage, with an FP32 offset and step per view beside them)
DTYPES = {"float32": torch.float32, "bfloat16": torch.bfloat16, "float16": torch.float16, "q16": torch.int16}


@dataclass(eq=False)
class Protocol:
    """Scan geometry and reconstruction shared by the jobs of one lane.

    ``scan`` carries the attributes of the reference ct_projector (nx, ny, nz,
    dx, dy, dz, cx, cy, cz, nu, nv, du, dv, off_u, off_v, dsd, dso); ``nz`` is
    the volume depth for cone protocols and ignored for fan/parallel, whose
    jobs bring 1..capacity slices each."""

    name: str
    kind: str  # "fan", "parallel" or "cone"
    algo: str  # "fbp" or "sqs"
    scan: object
    angles: Optional[np.ndarray] = None  # fan / parallel, float32 radians
    cone: Optional[Tuple[np.ndarray, ...]] = None  # (det_center, det_u, det_v, src), each [nview, 3]
    n_iter: int = 20
    beta: float = 0.0
    tv_weights: Tuple[float, float, float] = (1.0, 1.0, 1.0)  # (z, y, x)
    eps: float = 1e-8
    filter: str = "hann"
    storage: str = "float32"  # sinogram on the device
    image_storage: str = "float32"  # iterate as read by the forward projector

    def __post_init__(self):
        if self.kind not in ("fan", "parallel", "cone"):
            raise ValueError(f"unknown geometry kind {self.kind!r}")
        if self.algo not in ("fbp", "sqs"):
            raise ValueError(f"unknown algorithm {self.algo!r}")
        if self.kind == "cone" and self.algo != "sqs":
            raise ValueError("cone protocols reconstruct with SQS (there is no cone FBP)")
        if self.storage not in DTYPES:
            raise ValueError("storage must be float32, bfloat16, float16 or q16")
        if self.image_storage not in DTYPES or self.image_storage == "q16":
            raise ValueError("image_storage must be float32, bfloat16 or float16")

    @property
    def nview(self) -> int:
        return len(self.angles) if self.kind != "cone" else int(self.cone[0].shape[0])

    @property
    def slices_per_unit(self) -> int:
        return int(self.scan.nz) if self.kind == "cone" else 1

    def sinogram_shape(self, nz: int) -> Tuple[int, int, int, int]:
        """Host sinogram layout of a job with nz slices."""
        if self.kind == "cone":
            return (1, self.nview, int(self.scan.nv), int(self.scan.nu))
        return (nz, self.nview, 1, int(self.scan.nu))


@dataclass(eq=False)
class Job:
    """One reconstruction request.  ``sinogram`` is a host tensor of
    ``protocol.sinogram_shape(nz)`` in any float type, or a ``quant.Q16`` for
    q16 protocols (it is stored in the protocol's storage type on the device);
    ``arrival`` is in seconds from the start of the stream.  The server fills
    ``result`` ([nz, ny, nx] float32, host) and ``t_done``.

    ``deadline`` (seconds after arrival) bounds the wait of a client: a job not
    finished by then is cancelled with status "timeout".  ``resume`` continues
    an SQS job from a ``Snapshot`` taken by ``Engine.evict``.  ``status`` is
    one of new, queued, running, done, rejected (malformed), cancelled,
    timeout, evicted or failed (``error`` says why)."""

    job_id: int
    protocol: Protocol
    sinogram: torch.Tensor
    arrival: float = 0.0
    nz: int = 1
    result: Optional[torch.Tensor] = None
    t_admit: float = float("nan")
    t_done: float = float("nan")
    done_event: Optional[torch.cuda.Event] = field(default=None, repr=False)
    tag: object = None  # free for the caller (the synthetic streams record the data source)
    deadline: Optional[float] = None
    resume: Optional["Snapshot"] = field(default=None, repr=False)
    status: str = "new"
    error: Optional[str] = None

    @property
    def units(self) -> int:
        return 1 if self.protocol.kind == "cone" else self.nz

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


@dataclass(eq=False)
class Snapshot:
    """The state of an evicted SQS job: its iterate after ``done`` iterations
    (pinned host [units * slices per unit, ny, nx], valid once ``event`` has
    completed) and the job itself (protocol, sinogram, slices).  ``job()``
    makes the job that resumes it; the resumed job's result equals the
    uninterrupted one's."""

    source: Job
    x: torch.Tensor
    done: int
    event: torch.cuda.Event = field(repr=False)

    def ready(self) -> bool:
        return self.event.query()

    def job(self, arrival: float = 0.0, job_id: Optional[int] = None, deadline: Optional[float] = None) -> Job:
        j = self.source
        return Job(j.job_id if job_id is None else job_id, j.protocol, j.sinogram, arrival=arrival, nz=j.nz,
                   tag=j.tag, deadline=deadline, resume=self)


def _zlink_pattern(n: int) -> torch.Tensor:
    z = torch.zeros(n, dtype=torch.uint8)
    if n > 1:
        z[1:] |= 1
        z[:-1] |= 2
    return z


def _set_zlinks(z: torch.Tensor) -> None:
    """Device-side z links of one volume of len(z) slices (no host copy, so the
    lane's stream is not synchronised)."""
    n = z.numel()
    if n == 1:
        z.zero_()
        return
    z.fill_(3)
    z[:1].fill_(2)
    z[-1:].fill_(1)


# --------------------------------------------------------------------------- lanes
class Lane:
    """Device buffers, stream and slot pool of one protocol."""

    def __init__(self, engine: "Engine", protocol: Protocol, capacity: int):
        self.engine = engine
        self.p = protocol
        self.capacity = int(capacity)
        self.pool = SlotPool(self.capacity)
        self.dev = engine.device
        # one stream per lane (lanes overlap on the GPU), or the engine's one
        self.stream = engine.shared_stream if engine.shared_stream is not None else torch.cuda.Stream(self.dev)
        self.jobs: Dict[int, List] = {}  # job id -> [job, steps left]
        self.events: deque = deque()
        self.last_used = time.perf_counter()
        # launch sizes: exact up to 8 slices, then steps of 4 (fan/parallel); 1 volume (cone)
        self.granule = 1 if protocol.kind == "cone" else 4
        self.exact = 0 if protocol.kind == "cone" else 8
        s = protocol.scan
        self.ny, self.nx = int(s.ny), int(s.nx)
        if protocol.kind == "cone":
            self.geo = [torch.tensor(np.ascontiguousarray(a, dtype=np.float32), device=self.dev)
                        for a in protocol.cone]
        else:
            self.ang = torch.tensor(np.ascontiguousarray(protocol.angles, dtype=np.float32), device=self.dev)
            self.geom = _lib.GEOM_FAN if protocol.kind == "fan" else _lib.GEOM_PARALLEL

    @staticmethod
    def bytes_per_unit(p: Protocol) -> int:
        raise NotImplementedError

    @property
    def active(self) -> bool:
        return bool(self.jobs)

    def ready(self) -> bool:
        while self.events and self.events[0].query():
            self.events.popleft()
        return len(self.events) < 2

    def can_admit(self, job: Job) -> bool:
        return self.pool.fits(job.units)

    # sinogram buffers: y (storage dtype), plus per-view offsets and steps for q16
    def _alloc_sinogram(self, C: int, nview: int, nv: int, nu: int) -> None:
        p = self.p
        self.y = torch.zeros(C, nview, nv, nu, dtype=DTYPES[p.storage], device=self.dev)
        self.q16 = p.storage == "q16"
        self.ylo = torch.zeros(C, nview, device=self.dev) if self.q16 else None
        self.ystep = torch.zeros(C, nview, device=self.dev) if self.q16 else None

    def _ybufs(self) -> List[torch.Tensor]:
        return [self.y] + ([self.ylo, self.ystep] if self.q16 else [])

    def _ystored(self, b: int):
        """The first b slots of the sinogram as stored (Tensor or quant.Q16)."""
        return quant.Q16(self.y[:b], self.ylo[:b], self.ystep[:b]) if self.q16 else self.y[:b]

    def _load_sinogram(self, start: int, n: int, sino) -> None:
        """Copy a job's host sinogram into slots [start, start + n) (lane stream)."""
        dst = self.y[start:start + n]
        if self.q16:
            if not isinstance(sino, quant.Q16):
                raise TypeError(f"protocol {self.p.name} stores q16 sinograms: the job must bring a quant.Q16")
            dst.copy_(sino.code.reshape(dst.shape), non_blocking=True)
            self.ylo[start:start + n].copy_(sino.lo.reshape(n, -1), non_blocking=True)
            self.ystep[start:start + n].copy_(sino.step.reshape(n, -1), non_blocking=True)
        else:
            dst.copy_(sino.reshape(dst.shape), non_blocking=True)

    def _bufs(self) -> List[torch.Tensor]:
        """Per-slot device buffers that move with their jobs when slots are
        packed and are zeroed when freed."""
        return self._ybufs()

    def _release(self, job_ids: Sequence[int], old_hw: int) -> None:
        """Free the slots of ``job_ids`` (already removed from ``self.jobs``),
        pack the live slots to the front and zero the freed tail (lane stream)."""
        for jid in job_ids:
            self.pool.free(jid)
        with torch.cuda.stream(self.stream):
            self._apply_moves(self.pool.compact())
            new_hw = self.pool.high_water
            if new_hw < old_hw:
                for t in self._bufs():
                    t[new_hw:old_hw].zero_()
                self._clear_extra(new_hw, old_hw)

    def _clear_extra(self, lo: int, hi: int) -> None:
        pass

    def drop(self, job_id: int) -> Job:
        """Remove a running job without a result (cancellation, eviction)."""
        job = self.jobs.pop(job_id)[0]
        self._release([job_id], self.pool.high_water)
        self._record()
        return job

    @staticmethod
    def sinogram_bytes(p: Protocol, sino: int) -> int:
        """Device bytes of ``sino`` stored samples (q16 adds 8 bytes per view)."""
        extra = 8 * (sino // max(1, int(p.scan.nu) * (int(p.scan.nv) if p.kind == "cone" else 1)))
        return sino * DTYPES[p.storage].itemsize + (extra if p.storage == "q16" else 0)

    def _record(self):
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.events.append(ev)

    def release(self):
        self.stream.synchronize()


class SQSLane(Lane):
    """SQS-TV lane: slots are slices (fan/parallel) or volumes (cone)."""

    def __init__(self, engine, protocol, capacity):
        super().__init__(engine, protocol, capacity)
        p, s = protocol, protocol.scan
        C, U = self.capacity, p.slices_per_unit
        nview = p.nview
        nv = int(s.nv) if p.kind == "cone" else 1
        idt = DTYPES[p.image_storage]
        with torch.cuda.stream(self.stream):
            self._alloc_sinogram(C, nview, nv, int(s.nu))
            self.fp = torch.zeros(C, nview, nv, int(s.nu), device=self.dev)
            self.x = [torch.zeros(C, U, self.ny, self.nx, device=self.dev) for _ in range(2)]
            self.bp = torch.zeros(C, U, self.ny, self.nx, device=self.dev)
            self.xlp = ([torch.zeros(C, U, self.ny, self.nx, dtype=idt, device=self.dev) for _ in range(2)]
                        if idt != torch.float32 else None)
            if p.kind == "cone":
                self.zlink = _zlink_pattern(U).repeat(C).to(self.dev)
            else:
                self.zlink = torch.zeros(C, dtype=torch.uint8, device=self.dev)
            one = torch.ones(1, U, self.ny, self.nx, device=self.dev)
            self.norm = self._bp(self._fp(one)).reshape(U, self.ny, self.nx).contiguous()
        self.cur = 0
        self.graphs: Dict[Tuple[int, int], torch.cuda.CUDAGraph] = {}
        self.graph_pool = torch.cuda.graph_pool_handle() if engine.use_graphs else None

    @staticmethod
    def bytes_per_unit(p: Protocol) -> int:
        s = p.scan
        nv = int(s.nv) if p.kind == "cone" else 1
        sino = p.nview * nv * int(s.nu)
        img = p.slices_per_unit * int(s.ny) * int(s.nx)
        lp = 2 * DTYPES[p.image_storage].itemsize * img if p.image_storage != "float32" else 0
        # y, fp; x (2), bp, fp workspace (transposed image); captured graphs' workspaces
        return Lane.sinogram_bytes(p, sino) + sino * 4 + img * 4 * 4 + lp + sino * 4

    # projector calls on the lane stream (current stream inside the lane's context)
    def _fp(self, x, out=None):
        if self.p.kind == "cone":
            return D.siddon_fp(self.p.scan, x, *self.geo, out=out)
        return D.dd_fp(self.p.scan, x, self.ang, self.geom, out=out)

    def _bp(self, y, out=None):
        if self.p.kind == "cone":
            return D.siddon_bp(self.p.scan, y, *self.geo, out=out)
        return D.dd_bp(self.p.scan, y, self.ang, self.geom, out=out)

    def _iterate(self, b: int, src: int, dst: int):
        p = self.p
        xin = self.xlp[src][:b] if self.xlp is not None else self.x[src][:b]
        self._fp(xin, out=self.fp[:b])
        if self.q16:
            quant.sub_dequantized_(self.fp[:b], self._ystored(b))
        else:
            self.fp[:b].sub_(self.y[:b])
        self._bp(self.fp[:b], out=self.bp[:b])
        sqs_tv_update(self.x[src][:b], self.bp[:b], self.norm, p.beta, p.tv_weights, p.eps,
                      zlink=self.zlink[:b * p.slices_per_unit], out=self.x[dst][:b],
                      x_lp=self.xlp[dst][:b] if self.xlp is not None else None)

    def _run_step(self, b: int):
        src, dst = self.cur, 1 - self.cur
        key = (b, src)
        g = self.graphs.get(key)
        if g is not None:
            g.replay()
        else:
            # first step at this size runs eagerly (first-use allocations, kernel
            # attributes), then the same step is captured for the next time
            self._iterate(b, src, dst)
            if self.engine.use_graphs:
                g = torch.cuda.CUDAGraph()
                g.capture_begin(pool=self.graph_pool)
                try:
                    self._iterate(b, src, dst)
                finally:
                    g.capture_end()
                self.graphs[key] = g
        self.cur = dst

    def prepare(self) -> None:
        """Capture the iteration graphs of every launch size ahead of the
        stream.  The lane is empty, so every slot holds zeros and stays zero
        (a constant image has no TV terms)."""
        if self.jobs:
            raise RuntimeError("prepare() runs on an empty lane")
        with torch.cuda.stream(self.stream):
            for b in bucket_sizes(self.capacity, self.granule, self.exact):
                for _ in range(2):
                    self._run_step(b)

    def admit(self, job: Job) -> None:
        p = self.p
        start = self.pool.alloc(job.job_id, job.units)
        if start is None:  # fits only after packing
            self._apply_moves(self.pool.compact())
            start = self.pool.alloc(job.job_id, job.units)
        n = job.units
        snap = job.resume
        with torch.cuda.stream(self.stream):
            self._load_sinogram(start, n, job.sinogram)
            xs = self.x[self.cur][start:start + n]
            if snap is None:
                xs.zero_()
            else:  # continue from the snapshot's iterate
                xs.copy_(snap.x.reshape(xs.shape), non_blocking=True)
            if self.xlp is not None:
                self.xlp[self.cur][start:start + n].copy_(xs)
            if p.kind != "cone":
                _set_zlinks(self.zlink[start:start + n])
        self.jobs[job.job_id] = [job, p.n_iter - (snap.done if snap is not None else 0)]

    def _bufs(self) -> List[torch.Tensor]:
        return self._ybufs() + [self.x[self.cur]] + ([self.xlp[self.cur]] if self.xlp is not None else [])

    def _clear_extra(self, lo: int, hi: int) -> None:
        if self.p.kind != "cone":
            self.zlink[lo:hi].zero_()

    def _apply_moves(self, moves):
        if not moves:
            return
        with torch.cuda.stream(self.stream):
            bufs = self._bufs()
            for m in moves:
                for t in bufs:
                    t[m.dst:m.dst + m.n].copy_(t[m.src:m.src + m.n].clone())
                if self.p.kind != "cone":
                    self.zlink[m.dst:m.dst + m.n].copy_(self.zlink[m.src:m.src + m.n].clone())

    def snapshot(self, job_id: int) -> "Snapshot":
        """Copy a running job's current iterate to pinned host memory (lane
        stream) with its iteration count."""
        job, left = self.jobs[job_id]
        start, n = self.pool.range_of(job_id)
        x = torch.empty((n * self.p.slices_per_unit, self.ny, self.nx), pin_memory=True)
        with torch.cuda.stream(self.stream):
            x.copy_(self.x[self.cur][start:start + n].reshape(x.shape), non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        return Snapshot(job, x, self.p.n_iter - left, ev)

    def step(self) -> List[Job]:
        hw = self.pool.high_water
        b = bucket(hw, self.capacity, self.granule, self.exact)
        with torch.cuda.stream(self.stream):
            self._run_step(b)
        done = []
        for jid in list(self.jobs):
            rec = self.jobs[jid]
            rec[1] -= 1
            if rec[1] == 0:
                done.append(rec[0])
        if done:
            with torch.cuda.stream(self.stream):
                for job in done:
                    start, n = self.pool.range_of(job.job_id)
                    del self.jobs[job.job_id]
                    job.result = torch.empty((n * self.p.slices_per_unit, self.ny, self.nx), pin_memory=True)
                    job.result.copy_(self.x[self.cur][start:start + n].reshape(job.result.shape), non_blocking=True)
                    job.done_event = torch.cuda.Event()
                    job.done_event.record(self.stream)
            self._release([j.job_id for j in done], hw)
        self._record()
        self.last_used = time.perf_counter()
        return done


class FBPLane(Lane):
    """FBP lane (fan or parallel): each step filters and back projects every
    job admitted since the previous step as one batch of slices.  The ramp
    filter is built in FP64 (``exact``), so the result tracks the FP64
    reconstruction rather than the reference's FP32 filter construction."""

    def __init__(self, engine, protocol, capacity):
        super().__init__(engine, protocol, capacity)
        p, s = protocol, protocol.scan
        C = self.capacity
        with torch.cuda.stream(self.stream):
            self._alloc_sinogram(C, p.nview, 1, int(s.nu))
            self.img = torch.zeros(C, 1, self.ny, self.nx, device=self.dev)

    @staticmethod
    def bytes_per_unit(p: Protocol) -> int:
        s = p.scan
        sino = p.nview * int(s.nu)
        return Lane.sinogram_bytes(p, sino) + sino * 8 + int(s.ny) * int(s.nx) * 4

    def admit(self, job: Job) -> None:
        start = self.pool.alloc(job.job_id, job.units)
        if start is None:
            raise RuntimeError("FBP lane slots are freed every step; admission checked can_admit first")
        with torch.cuda.stream(self.stream):
            self._load_sinogram(start, job.units, job.sinogram)
        self.jobs[job.job_id] = [job, 1]

    def drop(self, job_id: int) -> Job:
        """Remove an admitted job before its step (its slots are zeroed and
        left as a hole for first-fit admission)."""
        job = self.jobs.pop(job_id)[0]
        start, n = self.pool.free(job_id)
        with torch.cuda.stream(self.stream):
            for t in self._ybufs():
                t[start:start + n].zero_()
        self._record()
        return job

    def prepare(self) -> None:
        """Run every launch size once on zeros (filter plans, workspaces)."""
        with torch.cuda.stream(self.stream):
            for b in bucket_sizes(self.capacity, self.granule, self.exact):
                self._filter_bp(b)

    def _filter_bp(self, b: int) -> None:
        p = self.p
        if self.q16:
            f = quant.ramp_filter(p.scan, self._ystored(b), p.filter, self.geom)
        else:
            y = self.y[:b] if self.y.dtype == torch.float32 else self.y[:b].float()
            f = D.ramp_filter(p.scan, y, p.filter, self.geom, exact=True)
        D.dd_bp(p.scan, f, self.ang, self.geom, is_fbp=True, out=self.img[:b])

    def step(self) -> List[Job]:
        b = bucket(self.pool.high_water, self.capacity, self.granule, self.exact)
        done = []
        with torch.cuda.stream(self.stream):
            self._filter_bp(b)
            for jid in list(self.jobs):
                job = self.jobs.pop(jid)[0]
                start, n = self.pool.free(jid)
                job.result = torch.empty((n, self.ny, self.nx), pin_memory=True)
                job.result.copy_(self.img[start:start + n].reshape(job.result.shape), non_blocking=True)
                job.done_event = torch.cuda.Event()
                job.done_event.record(self.stream)
                for t in self._ybufs():
                    t[start:start + n].zero_()
                done.append(job)
        self._record()
        self.last_used = time.perf_counter()
        return done


# --------------------------------------------------------------------------- engine
class Engine:
    """The server loop.  ``hbm_bytes`` bounds the lanes' buffers (default: 80%
    of the device memory free at start); ``capacity`` maps a protocol name to
    its lane's slot count (default 64 slices for fan/parallel lanes, as many
    cone volumes as a quarter of the budget holds, at most 4).

    Failures stay on the host and with the jobs they concern: a malformed job
    is rejected at ``submit``; ``cancel`` and a passed ``Job.deadline`` remove a
    queued or running job; a lane whose buffers cannot be allocated leaves its
    jobs queued and is retried after idle lanes are torn down (its jobs fail
    after ``max_alloc_retries`` failed attempts); an error raised by a lane's
    step fails that lane's jobs and tears the lane down while the other lanes
    go on.  ``faults`` (optional) is a host-side fault injector called as
    ``faults(event, protocol)`` before a lane is allocated ("lane_alloc") and
    before each lane step ("lane_step"); it may raise to simulate the failure
    of that operation."""

    def __init__(self, device=None, hbm_bytes: Optional[int] = None, max_wait: float = 1.0,
                 use_graphs: bool = True, capacity: Optional[Dict[str, int]] = None, slices_per_lane: int = 64,
                 track_busy: bool = False, faults=None, max_alloc_retries: int = 3, lane_streams: bool = False):
        if not torch.cuda.is_available():
            raise RuntimeError("the reconstruction server needs a CUDA device")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        _lib.lib()  # fail now, not at the first job, if the CUDA library is missing
        free, _ = torch.cuda.mem_get_info(self.device)
        self.budget = MemoryBudget(int(hbm_bytes) if hbm_bytes is not None else int(0.8 * free))
        self.queue = ArrivalQueue(max_wait)
        self.use_graphs = use_graphs
        self.capacity = dict(capacity or {})
        self.slices_per_lane = int(slices_per_lane)
        self.lanes: Dict[str, Lane] = {}
        self.jobs: Dict[int, Job] = {}
        self.retiring: List[Job] = []
        self.completed: List[Job] = []
        self.stats = LatencyStats()
        self.t0 = 0.0
        self.evictions = 0  # lanes torn down to make room for another protocol
        self.peak_reserved = 0
        self.track_busy = track_busy  # bracket every lane step with timing events (busy.BusyTracker)
        self.busy_tracker = None
        self.faults = faults
        self.max_alloc_retries = int(max_alloc_retries)
        # By default every lane enqueues on one stream: lanes take turns on
        # the GPU while the jobs of a lane share its launches.  Measured on the
        # B200 with 40 jobs of the mix with cone volumes: 4.84 recons/s against
        # 4.11 with one stream per lane (concurrent lanes slow each other's
        # kernels down more than they fill the GPU's gaps), and 27.0 against
        # 25.6 on the 150-job 2D stream.  lane_streams=True gives every lane
        # its own stream.
        self.shared_stream = None if lane_streams else torch.cuda.Stream(self.device)
        self.alloc_failures: Dict[str, int] = {}
        self.alloc_errors: Dict[str, str] = {}
        self.rejected: List[Job] = []
        self.cancelled: List[Job] = []  # cancelled, timed out or evicted
        self.failed: List[Job] = []

    # lanes ---------------------------------------------------------------
    def _lane_class(self, p: Protocol):
        return SQSLane if p.algo == "sqs" else FBPLane

    def _lane_capacity(self, p: Protocol) -> int:
        if p.name in self.capacity:
            return int(self.capacity[p.name])
        if p.kind == "cone":
            per = self._lane_class(p).bytes_per_unit(p)
            return int(max(1, min(4, self.budget.total // 4 // max(per, 1))))
        return self.slices_per_lane

    def lane_for(self, p: Protocol, units: int) -> Optional[Lane]:
        lane = self.lanes.get(p.name)
        if lane is not None:
            return lane
        cls = self._lane_class(p)
        cap = max(self._lane_capacity(p), units)
        need = cls.bytes_per_unit(p) * cap
        if need > self.budget.free:
            # tear down idle lanes, least recently used first
            for name, l in sorted(self.lanes.items(), key=lambda kv: kv[1].last_used):
                if need <= self.budget.free:
                    break
                if not l.active and all(e.query() for e in l.events):
                    l.release()
                    del self.lanes[name]
                    self.budget.release(name)
                    self.evictions += 1
        if not self.budget.try_reserve(p.name, need):
            return None
        self.peak_reserved = max(self.peak_reserved, self.budget.reserved)
        try:
            if self.faults is not None:
                self.faults("lane_alloc", p)
            lane = cls(self, p, cap)
        except (torch.cuda.OutOfMemoryError, _lib.CTProjectorError) as e:
            # leave the jobs queued; free what idle lanes hold before the retry
            self.budget.release(p.name)
            self.alloc_failures[p.name] = self.alloc_failures.get(p.name, 0) + 1
            self.alloc_errors[p.name] = f"{type(e).__name__}: {e}"
            self._teardown_idle()
            return None
        self.lanes[p.name] = lane
        return lane

    def _teardown_idle(self) -> None:
        for name, l in list(self.lanes.items()):
            if not l.active and all(e.query() for e in l.events):
                l.release()
                del self.lanes[name]
                self.budget.release(name)
                self.evictions += 1

    def warmup(self, protocols: Sequence[Protocol]) -> None:
        """Create the lanes of ``protocols`` ahead of the stream (normalisation
        images, filter plans, captured graphs of every launch size) so the
        first jobs do not pay for them."""
        for p in protocols:
            lane = self.lane_for(p, 1)
            if lane is not None and not lane.active:
                lane.prepare()
        torch.cuda.synchronize(self.device)

    # jobs ------------------------------------------------------------------
    def validate(self, job: Job) -> Optional[str]:
        """Why ``job`` cannot be served, or None."""
        p = job.protocol
        if job.job_id in self.jobs:
            return f"job id {job.job_id} is already in the server"
        if p.kind != "cone" and not (1 <= job.nz <= self._lane_capacity(p)):
            return f"{job.nz} slices: a {p.name} job brings 1 to {self._lane_capacity(p)} slices"
        shape = p.sinogram_shape(job.nz)
        sino = job.sinogram
        if p.storage == "q16":
            if not isinstance(sino, quant.Q16):
                return "a q16 protocol takes a quant.Q16 sinogram"
            if tuple(sino.code.shape) != shape or tuple(sino.lo.shape) != shape[:2] or \
                    tuple(sino.step.shape) != shape[:2]:
                return f"sinogram codes {tuple(sino.code.shape)} / offsets {tuple(sino.lo.shape)}, expected {shape}"
            if not (bool(torch.isfinite(sino.lo).all()) and bool(torch.isfinite(sino.step).all())):
                return "non-finite sinogram offsets or steps"
        else:
            if not isinstance(sino, torch.Tensor) or not sino.is_floating_point():
                return "the sinogram must be a floating-point tensor"
            if sino.numel() != int(np.prod(shape)):
                return f"sinogram of {tuple(sino.shape)}, expected {shape}"
        if job.resume is not None:
            if p.algo != "sqs" or job.resume.source.protocol.name != p.name:
                return "only an SQS job of the same protocol resumes from a snapshot"
            if not 0 <= job.resume.done < p.n_iter:
                return f"the snapshot has done {job.resume.done} of {p.n_iter} iterations"
        return None

    def submit(self, job: Job) -> bool:
        """Queue a job; a malformed one is rejected (status "rejected", the
        reason in ``error``) and False is returned."""
        why = self.validate(job)
        if why is not None:
            job.status, job.error = "rejected", why
            self.rejected.append(job)
            return False
        job.status = "queued"
        self.jobs[job.job_id] = job
        self.queue.push(Pending(job.arrival, job.job_id, job.protocol.name, job.units))
        return True

    def _remove(self, job: Job, status: str, error: Optional[str] = None) -> None:
        lane = self.lanes.get(job.protocol.name)
        if not self.queue.remove_job(job.job_id) and lane is not None and job.job_id in lane.jobs:
            lane.drop(job.job_id)
        del self.jobs[job.job_id]
        job.status, job.error = status, error
        (self.failed if status == "failed" else self.cancelled).append(job)

    def cancel(self, job_id: int, status: str = "cancelled") -> bool:
        """Remove a queued or running job without a result.  False if the job
        is not in the server or its result is already on its way."""
        job = self.jobs.get(job_id)
        if job is None or job.done_event is not None:
            return False
        self._remove(job, status)
        return True

    def evict(self, job_id: int) -> "Snapshot":
        """Take a running SQS job off the device: a snapshot of its iterate
        and iteration count (copied to pinned host memory on the lane's
        stream), from which ``Snapshot.job()`` resumes it later."""
        job = self.jobs.get(job_id)
        lane = self.lanes.get(job.protocol.name) if job is not None else None
        if lane is None or job_id not in lane.jobs or not isinstance(lane, SQSLane):
            raise ValueError(f"job {job_id} is not running in an SQS lane")
        snap = lane.snapshot(job_id)
        self._remove(job, "evicted")
        return snap

    def _expire(self, now: float) -> None:
        for job in list(self.jobs.values()):
            if job.deadline is not None and job.done_event is None and now - job.arrival > job.deadline:
                self._remove(job, "timeout", f"not finished {job.deadline:g} s after arrival")

    # loop ----------------------------------------------------------------
    def _admit(self, now: float) -> bool:
        admitted = False
        for item in self.queue.candidates(now, self.lanes.keys()):
            job = self.jobs[item.job_id]
            lane = self.lane_for(job.protocol, job.units)
            if lane is None:
                if self.alloc_failures.get(job.protocol.name, 0) > self.max_alloc_retries:
                    self._remove(job, "failed", "lane allocation failed: " + self.alloc_errors[job.protocol.name])
                continue
            if not lane.can_admit(job):
                continue
            lane.admit(job)
            job.status = "running"
            job.t_admit = now
            self.queue.remove(item)
            admitted = True
        return admitted

    def _step(self) -> bool:
        stepped = False
        for name, lane in list(self.lanes.items()):
            if lane.active and lane.ready():
                start = self.busy_tracker.begin(lane.stream) if self.busy_tracker is not None else None
                try:
                    if self.faults is not None:
                        self.faults("lane_step", lane.p)
                    self.retiring.extend(lane.step())
                except Exception as e:  # noqa: BLE001 -- isolate the failure to this lane's jobs
                    self._fail_lane(name, lane, f"{type(e).__name__}: {e}")
                    continue
                if start is not None:
                    self.busy_tracker.end(lane.stream, start)
                stepped = True
        return stepped

    def _fail_lane(self, name: str, lane: Lane, error: str) -> None:
        for jid in list(lane.jobs):
            job = lane.jobs.pop(jid)[0]
            del self.jobs[jid]
            job.status, job.error = "failed", error
            self.failed.append(job)
        lane.release()
        del self.lanes[name]
        self.budget.release(name)

    def _poll(self, now_fn) -> bool:
        finished = False
        still = []
        for job in self.retiring:
            if job.done_event.query():
                job.status = "done"
                job.t_done = now_fn()
                self.stats.add(job.latency, job.t_done)
                self.completed.append(job)
                del self.jobs[job.job_id]
                finished = True
            else:
                still.append(job)
        self.retiring = still
        return finished

    def busy(self) -> bool:
        return bool(self.jobs)

    def pass_once(self, now: float, now_fn=None) -> bool:
        """One pass of the server loop at time ``now`` (seconds on the caller's
        clock): admit queued jobs, step the lanes, collect finished results.
        Returns whether anything happened, so a caller driving the loop from
        its own event loop knows when to yield."""
        self._expire(now)
        progressed = self._admit(now)
        progressed |= self._step()
        progressed |= self._poll(now_fn or (lambda: now))
        return progressed

    def run(self, jobs: Sequence[Job], realtime: bool = True, idle_sleep: float = 1e-4) -> dict:
        """Serve ``jobs`` (sorted by arrival).  With ``realtime`` a job is
        offered only once its arrival time has passed on the wall clock;
        otherwise all are offered at once.  Returns the latency summary."""
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        if self.track_busy:
            self.busy_tracker = BusyTracker(self.device)
        self.t0 = time.perf_counter()
        now_fn = lambda: time.perf_counter() - self.t0  # noqa: E731
        while pending or self.busy():
            now = now_fn()
            while pending and (not realtime or pending[0].arrival <= now):
                self.submit(pending.popleft())
            progressed = self.pass_once(now, now_fn)
            if not progressed:
                time.sleep(idle_sleep)
        torch.cuda.synchronize(self.device)
        wall = time.perf_counter() - self.t0
        summary = self.stats.summary(0.0)
        if self.busy_tracker is not None:
            busy = self.busy_tracker.busy_seconds()
            summary.update(wall_s=wall, gpu_busy_s=busy, gpu_busy_frac=busy / wall if wall > 0 else 0.0)
            self.busy_tracker = None
        return summary

    def close(self) -> None:
        for name, lane in list(self.lanes.items()):
            lane.release()
            self.budget.release(name)
        self.lanes.clear()
