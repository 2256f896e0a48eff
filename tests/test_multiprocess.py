"""The multi-rank path on CPU with gloo, world size 2: every rank takes its
own batch or jobs (no data crosses ranks) and the reported time is the
slowest rank's.  Ranks are spawned processes; the rendezvous is on
127.0.0.1."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = torch.multiprocessing


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys

    import numpy as np
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.serving.scheduler import shard

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(10.0 + 5.0 * rank, torch.device("cpu"))
        # each rank's batch seed, and a checksum of a small phantom made from it
        rng = np.random.default_rng(S.seed_for(2, rank))
        img = S.ellipse_phantom(rng, 32, 32, 1.0, 1.0)
        mine = shard(list(range(11)), rank, world)
        q.put((rank, slowest, float(img.sum()), mine))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_and_disjoint_shards():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(world):
            rank, slowest, checksum, mine = q.get(timeout=120)
            out[rank] = (slowest, checksum, mine)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert out[0][0] == out[1][0] == 15.0  # both ranks report the slowest rank's time
    assert out[0][1] != out[1][1]  # independent batches
    a, b = out[0][2], out[1][2]
    assert sorted(a + b) == list(range(11)) and not set(a) & set(b)


def test_max_over_ranks_without_process_group():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    assert bench.max_over_ranks(3.5, torch.device("cpu")) == 3.5


def _view_split_worker(rank, world, port, q):
    import sys

    import numpy as np
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from ctprojector_b200.multigpu import gather_slabs, view_shares, view_split_bp

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        nview, m, shape = 7, 6, (5, 3, 4)
        rng = np.random.default_rng(0)  # the same operator and data on every rank
        mats = rng.standard_normal((nview, int(np.prod(shape)), m))
        prj = rng.standard_normal((nview, m))

        def bp_views(views):
            acc = np.zeros(int(np.prod(shape)))
            for v in views:
                acc += mats[v] @ prj[v]
            return torch.tensor(acc.reshape(shape), dtype=torch.float64)

        slab, (z0, z1) = view_split_bp(bp_views, nview)
        full = gather_slabs(slab, shape[0])
        ref = bp_views(range(nview))
        q.put((rank, view_shares(nview, rank, world), (z0, z1), float((slab - ref[z0:z1]).abs().max()),
               float((full - ref).abs().max())))
    finally:
        dist.destroy_process_group()


def test_view_split_back_projection_two_ranks():
    """Each rank back projects its share of the views; the reduce-scatter
    leaves it the sum over all views for its z slab, and the all-gather
    rebuilds the whole volume (5 slices over 2 ranks: uneven slabs)."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_view_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(world):
            rank, views, zr, err_slab, err_full = q.get(timeout=120)
            out[rank] = (views, zr, err_slab, err_full)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert sorted(out[0][0] + out[1][0]) == list(range(7)) and not set(out[0][0]) & set(out[1][0])
    assert out[0][1] == (0, 3) and out[1][1] == (3, 5)
    for r in range(world):
        assert out[r][2] <= 1e-12 and out[r][3] <= 1e-12


def test_view_shares_and_slabs_partition():
    """Round-robin view shares and z slabs cover every view and slice once,
    also with more ranks than slices (trailing ranks own empty slabs)."""
    from ctprojector_b200.multigpu import view_shares, z_slabs

    for nview, world in [(1, 1), (7, 2), (360, 8), (5, 8)]:
        shares = [view_shares(nview, r, world) for r in range(world)]
        assert sorted(v for s in shares for v in s) == list(range(nview))
    for nz, world in [(1, 1), (5, 2), (64, 8), (3, 8)]:
        slabs = z_slabs(nz, world)
        assert slabs[0][0] == 0 and slabs[-1][1] == nz
        assert all(a[1] == b[0] for a, b in zip(slabs, slabs[1:]))
        assert all(z1 >= z0 for z0, z1 in slabs)
    with pytest.raises(ValueError):
        view_shares(10, 2, 2)
