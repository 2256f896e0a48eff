"""View-split back projection over NCCL on the one GPU this process has
(world size 1): the split machinery around the Siddon back projector gives
the unsplit result.  The exchange itself with two ranks is tested on CPU
with gloo (test_multiprocess.py)."""
import socket

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_view_split_siddon_bp_single_rank():
    import torch.distributed as dist

    import cases
    from ctprojector_b200.multigpu import gather_slabs, view_split_bp
    from ctprojector_b200.projector import _device as D

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    name, p, inp = cases.case_siddon()
    geo = [torch.tensor(inp[k], device="cuda") for k in ("det_center", "det_u", "det_v", "src")]
    rng = np.random.default_rng(1)
    prj = torch.tensor(rng.uniform(0, 1, (1, geo[0].shape[0], p.nv, p.nu)).astype(np.float32), device="cuda")

    def bp_views(views):
        idx = torch.tensor(list(views), device="cuda", dtype=torch.long)
        g = [a.index_select(0, idx).contiguous() for a in geo]
        return D.siddon_bp(p, prj.index_select(1, idx).contiguous(), *g)[0]

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", rank=0, world_size=1, init_method=f"tcp://127.0.0.1:{port}",
                            device_id=torch.device("cuda", 0))
    try:
        slab, (z0, z1) = view_split_bp(bp_views, geo[0].shape[0])
        full = gather_slabs(slab, int(p.nz))
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    ref = D.siddon_bp(p, prj, *geo)[0]
    assert (z0, z1) == (0, int(p.nz))
    assert rel_l2(full.cpu().numpy(), ref.cpu().numpy()) <= 1e-6
