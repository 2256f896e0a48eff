"""ctp_dd2d_fp_noalloc: the forward projector for callers that cannot allocate
device memory at call time (their GPU memory belongs to another allocator, or
their service forbids allocation once running).  It takes its scratch from a
fixed array inside the library instead of a workspace or a pool, so its
output must equal ctp_dd2d_fp's on the same inputs, call after call.

Collected last on purpose: if it fails, a run that stops at the first failure
has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _geometry(nb, n, nview, nu, du, dx):
    from ctprojector_b200._lib import Geometry

    return Geometry(nb, n, n, 1, dx, dx, 1.0, 0.0, 0.0, 0.0, nu, 1, nview, du, 1.0, 0.0, 0.0, 1000.0, 500.0)


def _run_pair(geom_kind, g, img, ang):
    from ctprojector_b200._lib import lib

    L = lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    shape = (g.nbatch, g.nview, g.nv, g.nu)
    ws_bytes = L.ctp_dd2d_fp_workspace(ctypes.byref(g), geom_kind, 0, 0)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    ref = torch.empty(shape, dtype=torch.float32, device="cuda")
    rc = L.ctp_dd2d_fp(ctypes.c_void_p(ref.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                       ctypes.c_void_p(ang.data_ptr()), ctypes.byref(g), geom_kind, 0, 0,
                       ctypes.c_void_p(ws.data_ptr()), ws_bytes, stream)
    assert rc == 0
    outs = []
    for _ in range(2):  # two calls in a row share the fixed scratch
        out = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
        rc = L.ctp_dd2d_fp_noalloc(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                                   ctypes.c_void_p(ang.data_ptr()), ctypes.byref(g), geom_kind, 0, 0, stream)
        assert rc == 0
        outs.append(out)
    torch.cuda.synchronize()
    return ref.cpu().numpy(), [o.cpu().numpy() for o in outs]


@pytest.mark.parametrize("geom_kind", [0, 1])
def test_noalloc_matches_workspace_entry(geom_kind):
    rng = np.random.default_rng(20261203)
    nb, n, nview, nu = 2, 96, 60, 144
    du = 1.2858 / 1085.6 if geom_kind == 0 else 0.8
    g = _geometry(nb, n, nview, nu, du, 0.8)
    g.dsd, g.dso = (1085.6, 595.0) if geom_kind == 0 else (1000.0, 500.0)
    img = torch.tensor(rng.uniform(0, 0.03, (nb, 1, n, n)).astype(np.float32), device="cuda")
    ang = torch.tensor(np.sort(rng.uniform(0, 2 * np.pi, nview)).astype(np.float32), device="cuda")
    ref, outs = _run_pair(geom_kind, g, img, ang)
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    for out in outs:
        assert rel_l2(out, ref) <= TOL


def test_noalloc_second_call_with_other_geometry():
    """The fixed scratch keeps the previous call's contents; a call with a
    different geometry must not see them."""
    rng = np.random.default_rng(7)
    for n, nview, nu in ((64, 30, 100), (128, 90, 200)):
        g = _geometry(1, n, nview, nu, 0.7, 0.6)
        img = torch.tensor(rng.uniform(0, 0.03, (1, 1, n, n)).astype(np.float32), device="cuda")
        ang = torch.tensor(np.sort(rng.uniform(0, np.pi, nview)).astype(np.float32), device="cuda")
        ref, outs = _run_pair(1, g, img, ang)
        for out in outs:
            assert rel_l2(out, ref) <= TOL


def test_noalloc_rejects_requests_beyond_its_buffer():
    from ctprojector_b200._lib import CTP_ERR_TOO_LARGE, last_error_string, lib

    L = lib()
    cap = L.ctp_dd2d_fp_noalloc_capacity()
    assert cap == 32 << 20
    g = _geometry(1, 512, 720, 3000, 0.8, 0.8)  # 52 MB edge table alone
    assert L.ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0) > cap
    dummy = torch.empty(1, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    rc = L.ctp_dd2d_fp_noalloc(p, p, p, ctypes.byref(g), 1, 0, 0, None)
    assert rc == CTP_ERR_TOO_LARGE
    assert "scratch" in last_error_string()


def _scratch_allocations():
    from ctprojector_b200._lib import lib

    c = ctypes.c_ulonglong(0)
    assert lib().ctp_scratch_allocations(ctypes.byref(c)) == 0
    return c.value


def _noalloc_repeat(g, geom_kind, img, ang, calls=3):
    """ctp_dd2d_fp with the queried workspace, then `calls` noalloc calls:
    each must equal it, none may make a scratch allocation, and the device's
    free memory must not move between the last two."""
    from ctprojector_b200._lib import lib

    L = lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    shape = (g.nbatch, g.nview, g.nv, g.nu)
    ws_bytes = L.ctp_dd2d_fp_workspace(ctypes.byref(g), geom_kind, 0, 0)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    ref = torch.empty(shape, dtype=torch.float32, device="cuda")
    assert L.ctp_dd2d_fp(ctypes.c_void_p(ref.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                         ctypes.c_void_p(ang.data_ptr()), ctypes.byref(g), geom_kind, 0, 0,
                         ctypes.c_void_p(ws.data_ptr()), ws_bytes, stream) == 0
    outs = [torch.full(shape, float("nan"), dtype=torch.float32, device="cuda") for _ in range(calls)]
    torch.cuda.synchronize()
    allocs0 = _scratch_allocations()
    free = []
    for out in outs:
        assert L.ctp_dd2d_fp_noalloc(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                                     ctypes.c_void_p(ang.data_ptr()), ctypes.byref(g), geom_kind, 0, 0, stream) == 0
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    assert _scratch_allocations() == allocs0
    assert free[-2] == free[-1]
    r = ref.cpu().numpy()
    assert np.isfinite(r).all() and np.abs(r).max() > 0
    for out in outs:
        assert rel_l2(out.cpu().numpy(), r) <= TOL


def test_noalloc_chunked_stream_on_the_benchmark_stack():
    """The 16-slice 512 x 512 stack with 720 views of 768 cells: the full
    query (one chunk of 16 slices, 130 MB) exceeds the fixed 32 MiB, which
    holds the edge table and chunks of 2 slices' transposed images and line
    tables, so the call runs the streamed kernel in 8 chunks.  Three calls in
    a row equal ctp_dd2d_fp and allocate nothing."""
    from ctprojector_b200._lib import lib

    L = lib()
    rng = np.random.default_rng(98)
    nb, n, nview, nu = 16, 512, 720, 768
    g = _geometry(nb, n, nview, nu, 0.8, 0.8)
    assert L.ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0) > L.ctp_dd2d_fp_noalloc_capacity()
    img = torch.tensor(rng.uniform(0, 0.03, (nb, 1, n, n)).astype(np.float32), device="cuda")
    ang = torch.tensor((np.arange(nview) * np.pi / nview).astype(np.float32), device="cuda")
    _noalloc_repeat(g, 1, img, ang)


def test_noalloc_staged_path_allocates_nothing():
    """One 2048 x 2048 slice with 60 views of 2560 cells: its edge table and
    transposed image fit the fixed scratch but one slice's line tables
    (101 MB) do not, so the call runs the staged kernel (tables built per
    CTA in shared memory).  Three calls in a row equal ctp_dd2d_fp and
    allocate nothing."""
    from ctprojector_b200._lib import lib

    L = lib()
    rng = np.random.default_rng(99)
    nb, n, nview, nu = 1, 2048, 60, 2560
    g = _geometry(nb, n, nview, nu, 0.8, 0.8)
    assert L.ctp_dd2d_fp_workspace(ctypes.byref(g), 1, 0, 0) > L.ctp_dd2d_fp_noalloc_capacity()
    img = torch.tensor(rng.uniform(0, 0.03, (nb, 1, n, n)).astype(np.float32), device="cuda")
    ang = torch.tensor(np.sort(rng.uniform(0, np.pi, nview)).astype(np.float32), device="cuda")
    _noalloc_repeat(g, 1, img, ang)
