"""The streamed forward projector (line tables copied into shared memory by
bulk asynchronous copies) against the staged one on the same inputs, and the
device-side wait counter: every bounded mbarrier wait of the run completed."""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _fp(g, geom_kind, img, ang, ws_bytes):
    from ctprojector_b200._lib import lib

    L = lib()
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
    out = torch.full((g.nbatch, g.nview, g.nv, g.nu), float("nan"), device="cuda")
    rc = L.ctp_dd2d_fp(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                       ctypes.c_void_p(ang.data_ptr()), ctypes.byref(g), geom_kind, 0, 0,
                       ctypes.c_void_p(ws.data_ptr()), ws_bytes,
                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.ctpGetLastErrorString()
    return out


@pytest.mark.parametrize("geom_kind,n,nview,nu,du", [(0, 256, 360, 736, 1.2858 / 1085.6), (1, 200, 180, 300, 1.0),
                                                     (1, 96, 90, 130, 1.0), (0, 128, 40, 2300, 0.4 / 1085.6)])
def test_streamed_fp_equals_staged(geom_kind, n, nview, nu, du):
    from ctprojector_b200._lib import Geometry, lib

    # 8 slices: a stack that takes the streamed path
    g = Geometry(8, n, n, 1, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, nu, 1, nview, du, 1.0, 0.0, 0.0, 1085.6, 595.0)
    rng = np.random.default_rng(n)
    img = torch.tensor(rng.uniform(0, 1, (8, 1, n, n)).astype(np.float32), device="cuda")
    span = 2 * np.pi if geom_kind == 0 else np.pi
    ang = torch.tensor((np.arange(nview) * span / nview).astype(np.float32), device="cuda")
    full = lib().ctp_dd2d_fp_workspace(ctypes.byref(g), geom_kind, 0, 0)
    streamed = _fp(g, geom_kind, img, ang, full)
    # a workspace short of the line tables (but holding the rest) runs the staged kernel
    staged = _fp(g, geom_kind, img, ang, full - 256)
    torch.cuda.synchronize()
    assert rel_l2(streamed.cpu().numpy(), staged.cpu().numpy()) <= 1e-6


def test_no_bounded_wait_gave_up():
    from ctprojector_b200._lib import lib

    n = ctypes.c_uint(123)
    assert lib().ctp_wait_timeouts(ctypes.byref(n)) == 0
    assert n.value == 0
