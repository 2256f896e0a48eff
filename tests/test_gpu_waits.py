"""The streamed forward projector (line tables copied into shared memory by
bulk asynchronous copies), in one chunk of slices and in several, against the
staged one on the same inputs, and the device-side wait counter: every
bounded mbarrier wait of the run completed."""
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
    L = lib()
    full = L.ctp_dd2d_fp_workspace(ctypes.byref(g), geom_kind, 0, 0)
    streamed = _fp(g, geom_kind, img, ang, full)
    try:
        # the streamed path in chunks of 1 and 3 slices (3 + 3 + 2): the same
        # tables and sums per slice, so the same bits
        for cap in (1, 3):
            assert L.ctp_set_fp_stream_slices(cap) == 0
            chunked = _fp(g, geom_kind, img, ang, L.ctp_dd2d_fp_workspace(ctypes.byref(g), geom_kind, 0, 0))
            torch.cuda.synchronize()
            assert torch.equal(chunked, streamed), f"chunks of {cap} slices"
        # no streamed path: the staged kernel (tables built per CTA in shared memory)
        assert L.ctp_set_fp_stream_slices(0) == 0
        staged = _fp(g, geom_kind, img, ang, L.ctp_dd2d_fp_workspace(ctypes.byref(g), geom_kind, 0, 0))
    finally:
        assert L.ctp_set_fp_stream_slices(-1) == 0
    torch.cuda.synchronize()
    assert rel_l2(streamed.cpu().numpy(), staged.cpu().numpy()) <= 1e-6


def test_no_bounded_wait_gave_up():
    from ctprojector_b200._lib import lib

    n = ctypes.c_uint(123)
    assert lib().ctp_wait_timeouts(ctypes.byref(n)) == 0
    assert n.value == 0


def test_wait_that_gives_up_is_reported_and_writes_nothing():
    """Failure path of the bounded waits, on the GPU without a fault: with the
    first chunk wait's poll limit at 0 every CTA gives up at once, lets its
    in-flight copies land (full limit) and exits without writing.  The
    synchronous entry returns CTP_ERR_WAIT_TIMEOUT, the counter goes up, the
    output keeps its previous contents, and the context stays usable.  (Runs
    after test_no_bounded_wait_gave_up, which expects the counter at 0.)"""
    from ctprojector_b200._lib import CTP_ERR_WAIT_TIMEOUT, CTP_WAIT_POLLS_DEFAULT, Geometry, lib

    L = lib()
    nb, n, nview, nu = 2, 64, 40, 96
    da, dsd, dso = 1.2858 / 1085.6, 1085.6, 595.0
    g = Geometry(nb, n, n, 1, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, nu, 1, nview, da, 1.0, 0.0, 0.0, dsd, dso)
    rng = np.random.default_rng(11)
    img = torch.tensor(rng.uniform(0, 1, (nb, 1, n, n)).astype(np.float32), device="cuda")
    ang = torch.tensor((np.arange(nview) * 2 * np.pi / nview + 0.01).astype(np.float32), device="cuda")
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    F = ctypes.c_float

    def cupy_fp(out):
        return L.cupyDistanceDrivenFanProjection(P(out), P(img), P(ang), nb, n, n, 1, F(1.0), F(1.0), F(1.0),
                                                 F(0.0), F(0.0), F(0.0), nu, 1, nview, F(da), F(1.0), F(0.0),
                                                 F(0.0), F(dsd), F(dso), 0)

    def count():
        c = ctypes.c_uint(0)
        assert L.ctp_wait_timeouts(ctypes.byref(c)) == 0
        return c.value

    before = count()
    prj = torch.full((nb, nview, 1, nu), 7.0, device="cuda")
    assert L.ctp_set_wait_limit(0) == 0
    try:
        rc = cupy_fp(prj)
    finally:
        assert L.ctp_set_wait_limit(CTP_WAIT_POLLS_DEFAULT) == 0
    assert rc == CTP_ERR_WAIT_TIMEOUT, rc
    after = count()
    assert after > before
    torch.cuda.synchronize()
    assert bool(torch.all(prj == 7.0)), "a CTA whose wait gave up wrote output"

    # the context is usable and the default limit is back: the same call succeeds
    assert cupy_fp(prj) == 0
    assert count() == after
    ref = _fp(g, 0, img, ang, L.ctp_dd2d_fp_workspace(ctypes.byref(g), 0, 0, 0))
    torch.cuda.synchronize()
    assert rel_l2(prj.cpu().numpy(), ref.cpu().numpy()) == 0.0
