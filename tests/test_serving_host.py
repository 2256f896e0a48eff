"""Host-side policies of the reconstruction server (no GPU): slot ranges and
packing, launch buckets, the HBM budget, arrival order with aging, latency
statistics."""
import random

import pytest

from ctprojector_b200.serving.scheduler import (ArrivalQueue, LatencyStats, MemoryBudget, Pending, SlotPool, bucket,
                                                bucket_sizes)


def test_slot_pool_first_fit_and_free():
    pool = SlotPool(16)
    assert pool.alloc(1, 4) == 0
    assert pool.alloc(2, 8) == 4
    assert pool.alloc(3, 4) == 12
    assert pool.alloc(4, 1) is None
    pool.free(2)
    assert pool.used == 8 and pool.high_water == 16
    assert pool.alloc(5, 3) == 4  # first gap
    assert pool.alloc(6, 6) is None  # the gap left is 5 slots
    assert pool.fits(5) and not pool.fits(6)


def test_slot_pool_compact_moves_pack_in_order():
    pool = SlotPool(20)
    for j, n in ((1, 3), (2, 5), (3, 2), (4, 4)):
        pool.alloc(j, n)
    pool.free(1)
    pool.free(3)
    moves = pool.compact()
    assert [(m.job, m.src, m.dst, m.n) for m in moves] == [(2, 3, 0, 5), (4, 10, 5, 4)]
    assert pool.range_of(2) == (0, 5) and pool.range_of(4) == (5, 4)
    assert pool.high_water == pool.used == 9
    assert all(m.dst < m.src for m in moves)


def test_slot_pool_random_invariants():
    rng = random.Random(3)
    pool = SlotPool(64)
    live = {}
    for step in range(2000):
        if live and rng.random() < 0.45:
            j = rng.choice(list(live))
            pool.free(j)
            del live[j]
        else:
            n = rng.randint(1, 16)
            s = pool.alloc(step, n)
            if s is None and pool.fits(n):
                pool.compact()
                s = pool.alloc(step, n)
                assert s is not None
            if s is not None:
                live[step] = n
        if rng.random() < 0.1:
            pool.compact()
            assert pool.high_water == pool.used
        # ranges are disjoint and inside the pool
        spans = sorted(pool.range_of(j) for j in live)
        end = 0
        for s, n in spans:
            assert s >= end and s + n <= 64
            end = s + n
        assert pool.used == sum(live.values())


def test_slot_pool_rejects_bad_requests():
    pool = SlotPool(4)
    with pytest.raises(ValueError):
        pool.alloc(1, 5)
    pool.alloc(1, 2)
    with pytest.raises(ValueError):
        pool.alloc(1, 1)
    with pytest.raises(ValueError):
        SlotPool(0)


def test_bucket_sizes():
    assert [bucket(n, 64) for n in (0, 1, 2, 3, 5, 16, 17, 63, 64)] == [0, 1, 2, 3, 5, 16, 17, 63, 64]
    assert [bucket(n, 64, 4) for n in (1, 4, 5, 17, 61, 64)] == [4, 4, 8, 20, 64, 64]
    assert bucket(47, 46, 4) == 46
    assert bucket_sizes(10, 4) == [4, 8, 10]
    assert bucket_sizes(3) == [1, 2, 3]
    # exact small launches, then steps of the granule
    assert [bucket(n, 64, 4, 8) for n in (1, 3, 8, 9, 12, 13, 64)] == [1, 3, 8, 12, 12, 16, 64]
    assert bucket_sizes(20, 4, 8) == [1, 2, 3, 4, 5, 6, 7, 8, 12, 16, 20]


def test_memory_budget():
    b = MemoryBudget(100)
    assert b.try_reserve("a", 60)
    assert not b.try_reserve("b", 50)
    assert b.try_reserve("b", 40) and b.free == 0
    assert b.release("a") == 60 and b.free == 60
    with pytest.raises(ValueError):
        b.try_reserve("b", 1)


def test_arrival_queue_order_and_aging():
    q = ArrivalQueue(max_wait=1.0)
    q.push(Pending(0.3, 2, "fan", 1))
    q.push(Pending(0.1, 1, "cone", 1))
    q.push(Pending(0.2, 3, "par", 4))
    assert [p.job_id for p in q.candidates(0.5, {"fan", "par"})] == [1, 3, 2]
    # the head (cone) has waited 1 s: only jobs for other, existing lanes pass it
    assert [p.job_id for p in q.candidates(1.2, {"fan"})] == [1, 2]
    assert [p.job_id for p in q.candidates(1.2, {"fan", "par"})] == [1, 3, 2]
    q.remove(q.oldest())
    assert q.oldest().job_id == 3 and len(q) == 2


def test_latency_stats():
    st = LatencyStats()
    for i in range(100):
        st.add((i + 1) / 1000.0, 1.0 + i * 0.01)
    assert st.percentile(50) == pytest.approx(0.050)
    assert st.percentile(99) == pytest.approx(0.099)
    assert st.percentile(100) == pytest.approx(0.100)
    s = st.summary(0.0)
    assert s["jobs"] == 100
    assert s["recons_per_s"] == pytest.approx(100 / 1.99)
    assert s["p99_ms"] == pytest.approx(99.0)


def test_q16_storage_is_a_sinogram_format_only():
    import numpy as np

    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.serving import Protocol

    scan = S.Scan(32, 32, 1, 1.0, 1.0, 1.0, 48, 1, 1.0, 1.0, 10)
    ang = S.angles(10, np.pi)
    assert Protocol("p", "parallel", "sqs", scan, angles=ang, storage="q16").storage == "q16"
    with pytest.raises(ValueError):
        Protocol("p", "parallel", "sqs", scan, angles=ang, image_storage="q16")
    with pytest.raises(ValueError):
        Protocol("p", "parallel", "sqs", scan, angles=ang, storage="int8")


def test_q16_host_values_and_slices():
    import torch

    from ctprojector_b200.quant import Q16

    code = torch.tensor([[[[0, -1, 32767, 2]]], [[[5, 6, 7, 8]]]], dtype=torch.int16)  # -1 is code 65535
    lo = torch.tensor([[1.0], [-2.0]])
    step = torch.tensor([[0.5], [0.25]])
    q = Q16(code, lo, step)
    v = q.float()
    assert v.dtype == torch.float32 and tuple(v.shape) == (2, 1, 1, 4)
    assert v[0, 0, 0].tolist() == [1.0, 1.0 + 0.5 * 65535, 1.0 + 0.5 * 32767, 2.0]
    assert v[1, 0, 0].tolist() == [-2.0 + 0.25 * k for k in (5, 6, 7, 8)]
    one = q[1:]
    assert tuple(one.shape) == (1, 1, 1, 4) and tuple(one.lo.shape) == (1, 1)
    assert one.nbytes == 4 * 2 + 2 * 4


def test_arrival_queue_removes_a_job_by_id():
    q = ArrivalQueue(1.0)
    for i, t in enumerate([0.3, 0.1, 0.2]):
        q.push(Pending(t, i, "lane", 1))
    assert q.remove_job(2) and not q.remove_job(2)
    assert [p.job_id for p in q.candidates(0.5)] == [1, 0]
    assert not q.remove_job(7) and len(q) == 2
