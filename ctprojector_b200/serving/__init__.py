"""Continuous-batching reconstruction server (engine) and its host-side
policies (scheduler); ``per_call`` is the plain one-call-per-operation path
it is measured against."""
from .engine import DTYPES, Engine, FBPLane, Job, Lane, Protocol, SQSLane
from .scheduler import ArrivalQueue, LatencyStats, MemoryBudget, Move, Pending, SlotPool, bucket, bucket_sizes

__all__ = ["DTYPES", "Engine", "FBPLane", "Job", "Lane", "Protocol", "SQSLane", "ArrivalQueue", "LatencyStats",
           "MemoryBudget", "Move", "Pending", "SlotPool", "bucket"]
