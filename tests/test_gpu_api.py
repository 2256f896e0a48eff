"""GPU behaviour of the public API and the C ABI: host-pointer (c*) vs
device-pointer (cupy*) entries, output semantics, determinism, edge cases,
error reporting and reduced-precision storage."""
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


def _case(name):
    import cases

    for fn in cases.ALL:
        n, p, inp = fn()
        if n == name:
            return p, inp
    raise KeyError(name)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().float().cpu().numpy()


@pytest.mark.parametrize("fan", [True, False])
def test_numpy_module_equals_device_module(fan):
    from ctprojector_b200.projector.cupy import fan_equiangular as CF, parallel as CP
    from ctprojector_b200.projector.numpy import fan_equiangluar as NF, parallel as NP

    p, inp = _case("fan_basic" if fan else "par_basic")
    C, N = (CF, NF) if fan else (CP, NP)
    prj_n = N.distance_driven_fp(p, inp["img"], inp["angles"])
    prj_c = host(C.distance_driven_fp(p, dev(inp["img"]), dev(inp["angles"])))
    np.testing.assert_array_equal(prj_n, prj_c)
    bp_n = N.distance_driven_bp(p, prj_n, inp["angles"], True)
    bp_c = host(C.distance_driven_bp(p, dev(prj_n), dev(inp["angles"]), True))
    np.testing.assert_array_equal(bp_n, bp_c)
    f_n = N.ramp_filter(p, prj_n, "hann")
    f_c = host(C.ramp_filter(p, dev(prj_n), "hann"))
    np.testing.assert_allclose(f_n, f_c, rtol=0, atol=1e-6 * np.abs(f_c).max())


@pytest.mark.parametrize("nb,nview", [(6, 500), (11, 900)])
def test_host_entries_large_arrays_through_pinned_staging(nb, nview):
    """Host arrays above the staging threshold cross the link in 8 MB pinned
    chunks (worker threads copy the pageable side; 12 and 26 MB sinograms,
    ragged last chunks): the results have the same bits as the device
    entries, from pageable and from pinned host arrays."""
    from ctprojector_b200.projector.cupy import parallel as CP
    from ctprojector_b200.projector.numpy import parallel as NP
    from cases import Proj

    p = Proj(nx=400, ny=400, nz=1, dx=1.0, dy=1.0, nu=700, nv=1, du=0.9, dv=1.0, nview=nview)
    rng = np.random.default_rng(21)
    img = rng.uniform(0, 1, (nb, 1, 400, 400)).astype(np.float32)
    ang = (np.arange(nview) * np.pi / nview).astype(np.float32)
    prj_c = host(CP.distance_driven_fp(p, dev(img), dev(ang)))
    assert prj_c.nbytes > 8 << 20 and prj_c.nbytes % (8 << 20) != 0
    np.testing.assert_array_equal(NP.distance_driven_fp(p, img, ang), prj_c)
    pinned = torch.empty(img.shape, dtype=torch.float32, pin_memory=True)
    pinned.numpy()[:] = img
    np.testing.assert_array_equal(NP.distance_driven_fp(p, pinned.numpy(), ang), prj_c)
    bp_c = host(CP.distance_driven_bp(p, dev(prj_c), dev(ang)))
    np.testing.assert_array_equal(NP.distance_driven_bp(p, prj_c, ang), bp_c)
    f_c = host(CP.ramp_filter(p, dev(prj_c), "hann"))
    np.testing.assert_allclose(NP.ramp_filter(p, prj_c, "hann"), f_c, rtol=0, atol=1e-6 * np.abs(f_c).max())


def test_reference_device_entry_accumulates_like_reference():
    """cupyDistanceDrivenParallelBackprojection adds into the image (the
    reference zero-fills in the Python wrapper, not in C)."""
    from ctprojector_b200._lib import lib

    p, inp = _case("par_basic")
    prj = dev(np.ones([1, 90, 1, 96], np.float32))
    ang = dev(inp["angles"])
    img = torch.full([1, 1, 64, 64], 2.0, device="cuda")
    args = [ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(prj.data_ptr()), ctypes.c_void_p(ang.data_ptr()),
            1, 64, 64, 1, 0.8, 0.8, 1.0, 0.0, 0.0, 0.0, 96, 1, 90, 0.8, 1.0, 0.0, 0.0, 1]
    assert lib().cupyDistanceDrivenParallelBackprojection(*args) == 0
    first = host(img).copy()
    assert lib().cupyDistanceDrivenParallelBackprojection(*args) == 0
    second = host(img)
    np.testing.assert_allclose(second - 2.0, 2 * (first - 2.0), rtol=1e-6, atol=1e-5)


@pytest.mark.parametrize("op", ["fp", "bp", "adj", "filter", "filter_exact"])
def test_gather_kernels_are_deterministic(op):
    from ctprojector_b200.projector.cupy import fan_equiangular as F

    p, inp = _case("fan_basic")
    img, ang = dev(inp["img"]), dev(inp["angles"])
    prj = F.distance_driven_fp(p, img, ang)
    fn = {
        "fp": lambda: F.distance_driven_fp(p, img, ang),
        "bp": lambda: F.distance_driven_bp(p, prj, ang),
        "adj": lambda: F.distance_driven_bp(p, prj, ang, adjoint=True),
        "filter": lambda: F.ramp_filter(p, prj),
        "filter_exact": lambda: F.ramp_filter(p, prj, exact=True),
    }[op]
    a, b = host(fn()), host(fn())
    assert np.array_equal(a, b)


# The Siddon back projectors scatter with FP32 atomics (as the reference's
# SiddonRayTracingTransposeAtomicAdd does), so the order of the additions into
# a voxel changes from run to run.  Bounded: relative L2 between runs, and the
# largest voxel difference against the largest voxel (a few FP32 roundings).
SIDDON_RUN_TO_RUN = 1e-6
SIDDON_RUN_TO_RUN_MAX = 4e-6


@pytest.mark.parametrize("kind", ["cone", "fan"])
def test_siddon_bp_run_to_run_difference_is_bounded(kind):
    from ctprojector_b200.projector.cupy import cone as C
    from ctprojector_b200.projector.cupy import fan_equiangular as F

    if kind == "cone":
        p, inp = _case("siddon")
        geo = [dev(inp[k]) for k in ("det_center", "det_u", "det_v", "src")]
        prj = C.siddon_fp_arbitrary(p, dev(inp["img"]), *geo)
        fn = lambda: C.siddon_bp_arbitrary(p, prj, *geo)  # noqa: E731
    else:
        p, inp = _case("fan_basic")
        ang = dev(inp["angles"])
        prj = F.siddon_fp(p, dev(inp["img"]), ang)
        fn = lambda: F.siddon_bp(p, prj, ang)  # noqa: E731
    runs = [host(fn()).astype(np.float64) for _ in range(4)]
    scale = np.abs(runs[0]).max()
    for r in runs[1:]:
        assert rel_l2(r, runs[0]) <= SIDDON_RUN_TO_RUN
        assert np.abs(r - runs[0]).max() <= SIDDON_RUN_TO_RUN_MAX * scale


def test_ragged_sizes_and_batch(oracle):
    """Sizes that are not multiples of the tiles, batch 3."""
    from cases import Proj
    from ctprojector_b200.projector.cupy import parallel as P

    p = Proj(nx=37, ny=23, nz=1, dx=0.9, dy=1.1, nu=45, nv=1, du=0.85, dv=1.0, off_u=0.2)
    rng = np.random.default_rng(11)
    img = rng.uniform(0, 1, [3, 1, 23, 37]).astype(np.float32)
    ang = np.sort(rng.uniform(0, np.pi, 17)).astype(np.float32)
    prj = host(P.distance_driven_fp(p, dev(img), dev(ang)))
    assert rel_l2(prj, oracle.dd_fp(p, img, ang, "parallel")) <= 1e-5
    bp = host(P.distance_driven_bp(p, dev(prj), dev(ang)))
    assert rel_l2(bp, oracle.dd_bp(p, prj, ang, "parallel")) <= 1e-5


def test_empty_batch_is_noop():
    from ctprojector_b200.projector.cupy import parallel as P

    p, inp = _case("par_basic")
    out = P.distance_driven_fp(p, torch.zeros([0, 1, 64, 64], device="cuda"), dev(inp["angles"]))
    assert tuple(out.shape) == (0, 90, 1, 96)


def test_invalid_geometry_raises():
    from ctprojector_b200.errors import CTProjectorError
    from ctprojector_b200.projector.cupy import parallel as P

    p, inp = _case("par_basic")
    p.nu = 0
    with pytest.raises(CTProjectorError) as e:
        P.distance_driven_fp(p, dev(inp["img"]), dev(inp["angles"]))
    assert e.value.code == 1001


def test_non_strict_mode_prints_and_returns(capsys):
    from ctprojector_b200 import errors
    from ctprojector_b200.projector.cupy import parallel as P

    p, inp = _case("par_basic")
    p.nu = 0
    errors.set_strict(False, thread_local=True)
    try:
        P.distance_driven_fp(p, dev(inp["img"]), dev(inp["angles"]))
    finally:
        errors.set_strict(True, thread_local=True)
    assert "1001" in capsys.readouterr().out


@pytest.mark.parametrize("dt", ["bfloat16", "float16"])
def test_low_precision_storage(dt, oracle):
    """BF16/FP16 storage with FP32 accumulation: error against the FP64 oracle
    stays at the storage rounding level."""
    from ctprojector_b200.projector.cupy import fan_equiangular as F

    p, inp = _case("fan_basic")
    tdt = getattr(torch, dt)
    ang = dev(inp["angles"])
    img16 = dev(inp["img"]).to(tdt)
    prj = F.distance_driven_fp(p, img16, ang, dtype=tdt)
    assert prj.dtype == tdt
    ref = oracle.dd_fp(p, host(img16), inp["angles"], "fan")
    tol = 4e-3 if dt == "bfloat16" else 5e-4
    assert rel_l2(host(prj), ref) <= tol
    bp = F.distance_driven_bp(p, prj, ang, adjoint=True)
    ref_bp = oracle.dd_bp(p, host(prj), inp["angles"], "fan", adjoint=True)
    assert rel_l2(host(bp), ref_bp) <= 1e-5


def test_nnz_matches_oracle(oracle):
    from ctprojector_b200.projector import _device as D

    for name in ("fan_basic", "par_offsets"):
        p, inp = _case(name)
        geom = 0 if name.startswith("fan") else 1
        n = D.dd_nnz(p, dev(inp["angles"]), geom, inp["img"].shape[1:])
        assert n == oracle.dd_nnz(p, inp["angles"], "fan" if geom == 0 else "parallel", inp["img"].shape[1:])
    p, inp = _case("siddon")
    a = [inp[k] for k in ("det_center", "det_u", "det_v", "src")]
    n = D.siddon_nnz(p, *[dev(v) for v in a], image_shape=inp["img"].shape[1:])
    assert abs(n - oracle.siddon_nnz(p, *a, shape=inp["img"].shape[1:])) <= 1e-4 * n
