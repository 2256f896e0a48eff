"""Continuous-batching reconstruction server (engine) and its host-side
policies (scheduler); ``per_call`` is the plain one-call-per-operation path
it is measured against, ``mix`` the served protocols and arrival streams.

The engine symbols are imported on first use, so that the pure modules
(``mix``, ``scheduler``) can be imported without loading the projector
library."""
import importlib

_ENGINE = ("DTYPES", "Engine", "FBPLane", "Job", "Lane", "Protocol", "SQSLane")
_SCHEDULER = ("ArrivalQueue", "LatencyStats", "MemoryBudget", "Move", "Pending", "SlotPool", "bucket",
              "bucket_sizes")

__all__ = list(_ENGINE + _SCHEDULER)


def __getattr__(name):
    if name in _ENGINE:
        return getattr(importlib.import_module(".engine", __name__), name)
    if name in _SCHEDULER:
        return getattr(importlib.import_module(".scheduler", __name__), name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
