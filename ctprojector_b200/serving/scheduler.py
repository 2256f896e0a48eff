"""Host-side bookkeeping of the reconstruction server: slot ranges inside a
lane, the HBM budget, the arrival queue and latency statistics.

Nothing here touches the GPU, so the policies are unit-tested on the CPU; the
engine (``engine.py``) executes what they decide (copies, kernel launches) on
the lanes' CUDA streams.
"""
from __future__ import annotations

import bisect
from collections import OrderedDict
from dataclasses import dataclass, field
from typing import Dict, Iterator, List, Optional, Tuple


# --------------------------------------------------------------------------- slots
@dataclass(frozen=True)
class Move:
    """Copy ``n`` slots of ``job`` from ``src`` to ``dst`` (``dst < src``)."""

    job: int
    src: int
    dst: int
    n: int


class SlotPool:
    """Slots 0 .. capacity-1 of one lane, handed out as contiguous ranges.

    Kernels run over slots [0, high_water), so holes left by finished jobs
    cost work until ``compact`` closes them; it returns the moves that pack the
    live ranges to the front in their current order."""

    def __init__(self, capacity: int):
        if capacity <= 0:
            raise ValueError("capacity must be positive")
        self.capacity = int(capacity)
        self._ranges: "OrderedDict[int, Tuple[int, int]]" = OrderedDict()  # job -> (start, n), by start

    def _sorted(self) -> List[Tuple[int, int, int]]:
        return sorted(((s, n, j) for j, (s, n) in self._ranges.items()))

    def alloc(self, job: int, n: int) -> Optional[int]:
        """First-fit range of ``n`` slots for ``job``; None if no gap is large enough."""
        if n <= 0 or n > self.capacity:
            raise ValueError(f"cannot allocate {n} slots of {self.capacity}")
        if job in self._ranges:
            raise ValueError(f"job {job} already holds slots")
        pos = 0
        for s, m, _ in self._sorted():
            if s - pos >= n:
                break
            pos = s + m
        if pos + n > self.capacity:
            return None
        self._ranges[job] = (pos, n)
        return pos

    def free(self, job: int) -> Tuple[int, int]:
        return self._ranges.pop(job)

    def range_of(self, job: int) -> Tuple[int, int]:
        return self._ranges[job]

    def jobs(self) -> List[int]:
        return [j for _, _, j in self._sorted()]

    @property
    def used(self) -> int:
        return sum(n for _, n in self._ranges.values())

    @property
    def high_water(self) -> int:
        return max((s + n for s, n in self._ranges.values()), default=0)

    def fits(self, n: int) -> bool:
        """Whether ``alloc(n)`` would succeed now or after ``compact``."""
        return self.used + n <= self.capacity

    def compact(self) -> List[Move]:
        moves = []
        pos = 0
        for s, n, j in self._sorted():
            if s != pos:
                moves.append(Move(j, s, pos, n))
                self._ranges[j] = (pos, n)
            pos += n
        return moves


def bucket(n: int, capacity: int, granule: int = 1, exact: int = 0) -> int:
    """Launch size for ``n`` live slots: ``n`` itself up to ``exact``, above
    that rounded up to a multiple of ``granule``; at most ``capacity``.  One
    graph is captured per size, so the granule bounds the number of graphs;
    empty slots in a launch are work done on zeros, which ``exact`` spares the
    small launches (a lone one-slice job runs one slice, not ``granule``)."""
    if n <= 0:
        return 0
    if n <= exact:
        return min(n, capacity)
    g = max(1, int(granule))
    return min(-(-n // g) * g, capacity)


def bucket_sizes(capacity: int, granule: int = 1, exact: int = 0):
    """Every launch size ``bucket`` can return for this capacity."""
    return sorted({bucket(n, capacity, granule, exact) for n in range(1, capacity + 1)})


# --------------------------------------------------------------------------- memory
class MemoryBudget:
    """Bytes of HBM the server may hold; lanes reserve their buffers here
    before allocating them and release them when they are torn down."""

    def __init__(self, total_bytes: int):
        self.total = int(total_bytes)
        self._held: Dict[object, int] = {}

    @property
    def reserved(self) -> int:
        return sum(self._held.values())

    @property
    def free(self) -> int:
        return self.total - self.reserved

    def try_reserve(self, key, nbytes: int) -> bool:
        if key in self._held:
            raise ValueError(f"{key!r} already holds a reservation")
        if nbytes > self.free:
            return False
        self._held[key] = int(nbytes)
        return True

    def release(self, key) -> int:
        return self._held.pop(key, 0)


# --------------------------------------------------------------------------- arrivals
@dataclass(order=True)
class Pending:
    arrival: float
    job_id: int
    lane_key: object = field(compare=False)
    units: int = field(compare=False)


class ArrivalQueue:
    """Jobs that arrived and wait for a slot, in arrival order.

    ``candidates`` yields them oldest first.  Once the oldest job has waited
    ``max_wait`` seconds it becomes a barrier: jobs behind it are offered only
    if they go to a lane other than the one it waits for and that lane already
    exists, so a large job is not starved by a stream of small ones while
    memory is freed for it."""

    def __init__(self, max_wait: float = 1.0):
        self.max_wait = float(max_wait)
        self._q: List[Pending] = []

    def __len__(self) -> int:
        return len(self._q)

    def push(self, item: Pending) -> None:
        bisect.insort(self._q, item)

    def remove(self, item: Pending) -> None:
        self._q.remove(item)

    def remove_job(self, job_id: int) -> bool:
        """Drop a queued job by id (cancellation); False if it is not queued."""
        for i, item in enumerate(self._q):
            if item.job_id == job_id:
                del self._q[i]
                return True
        return False

    def oldest(self) -> Optional[Pending]:
        return self._q[0] if self._q else None

    def candidates(self, now: float, existing_lanes=()) -> Iterator[Pending]:
        if not self._q:
            return
        head = self._q[0]
        starving = now - head.arrival >= self.max_wait
        for item in list(self._q):
            if starving and item is not head:
                if item.lane_key == head.lane_key or item.lane_key not in existing_lanes:
                    continue
            yield item


# --------------------------------------------------------------------------- statistics
class LatencyStats:
    """Per-job latencies (seconds) and completion times."""

    def __init__(self):
        self.latency: List[float] = []
        self.done_at: List[float] = []

    def add(self, latency: float, done_at: float) -> None:
        self.latency.append(float(latency))
        self.done_at.append(float(done_at))

    def __len__(self) -> int:
        return len(self.latency)

    def percentile(self, p: float) -> float:
        """Nearest-rank percentile (p in [0, 100])."""
        if not self.latency:
            return float("nan")
        xs = sorted(self.latency)
        k = max(0, min(len(xs) - 1, int(-(-p * len(xs) // 100)) - 1))
        return xs[k]

    def throughput(self, t_start: float) -> float:
        """Completed jobs per second from ``t_start`` to the last completion."""
        if not self.done_at:
            return 0.0
        span = max(self.done_at) - t_start
        return len(self.done_at) / span if span > 0 else float("inf")

    def summary(self, t_start: float) -> dict:
        return {"jobs": len(self), "recons_per_s": self.throughput(t_start),
                "p50_ms": 1e3 * self.percentile(50), "p99_ms": 1e3 * self.percentile(99),
                "max_ms": 1e3 * max(self.latency) if self.latency else float("nan")}


def shard(items, rank: int, world: int):
    """Round-robin share of ``items`` for one of ``world`` replicas (one server
    per GPU; jobs are independent, so no data crosses ranks)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return [x for i, x in enumerate(items) if i % world == rank]
