"""GPU-busy time of a serving run from CUDA events.

Each unit of device work (one lane step of the server, one job of the
per-call path) is bracketed by two timing events recorded on the stream that
runs it.  After the run every event is placed on one time axis (elapsed time
from an origin event recorded when tracking starts) and the union of the
intervals is the time the GPU had work of this run in flight; lanes that run
concurrently on several streams are counted once.  busy / wall says how much
room scheduling had left: a path whose GPU is already busy most of the wall
time cannot be made much faster by batching its launches."""
from __future__ import annotations

from typing import List, Tuple

import torch


class BusyTracker:
    def __init__(self, device=None):
        self.device = device
        self.origin = torch.cuda.Event(enable_timing=True)
        self.origin.record(torch.cuda.current_stream(device))
        self.intervals: List[Tuple[torch.cuda.Event, torch.cuda.Event]] = []

    def begin(self, stream) -> torch.cuda.Event:
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        return ev

    def end(self, stream, start: torch.cuda.Event) -> None:
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        self.intervals.append((start, ev))

    def busy_seconds(self) -> float:
        """Union of the recorded intervals, in seconds (synchronises)."""
        torch.cuda.synchronize(self.device)
        spans = sorted((self.origin.elapsed_time(a), self.origin.elapsed_time(b)) for a, b in self.intervals)
        total, cur_a, cur_b = 0.0, None, None
        for a, b in spans:
            if cur_b is None or a > cur_b:
                if cur_b is not None:
                    total += cur_b - cur_a
                cur_a, cur_b = a, b
            else:
                cur_b = max(cur_b, b)
        if cur_b is not None:
            total += cur_b - cur_a
        return total * 1e-3
