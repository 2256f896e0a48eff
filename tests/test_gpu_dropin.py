"""Drop-in: the reference's own, unmodified Python modules running on libctp.so.

The reference package (ct_projector, installed offline into baseline/_ref from
its source tree, git-ignored) loads its CUDA library from
ct_projector/kernel/bin/libprojector.so and its prior from libprior.so through
pkg_resources (projector/numpy/parallel.py:14-16 and the other modules).  The
test copies the installed package into a temporary directory, puts
ctprojector_b200/libctp.so in both library slots, imports the reference's
numpy modules from there and runs their public functions on the golden cases:
their results equal this repository's own numpy modules (the same entries,
called by the reference's ctypes code) and match the reference library's own
outputs (the golden fixtures) within the parity bar.  The reference's cupy
modules need cupy, which this environment does not have.
"""
import importlib
import os
import shutil
import sys

import numpy as np
import pytest

from conftest import ROOT, load_golden, rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-5
REF_PKG = os.path.join(ROOT, "baseline", "_ref", "ct_projector")
LIBCTP = os.path.join(ROOT, "ctprojector_b200", "libctp.so")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def ref(tmp_path_factory):
    """The reference's numpy modules, imported from a copy whose library slots
    hold libctp.so."""
    if not os.path.isdir(REF_PKG):
        pytest.skip("the reference package is not installed in baseline/_ref")
    if not os.path.exists(LIBCTP):
        pytest.fail("libctp.so is not built")
    root = tmp_path_factory.mktemp("dropin")
    pkg = root / "ct_projector"
    shutil.copytree(REF_PKG, pkg, ignore=shutil.ignore_patterns("__pycache__"))
    (pkg / "kernel" / "bin").mkdir(parents=True)
    for name in ("libprojector.so", "libprior.so"):
        os.symlink(LIBCTP, pkg / "kernel" / "bin" / name)
    sys.path.insert(0, str(root))
    try:
        mods = {n: importlib.import_module(f"ct_projector.projector.numpy.{n}")
                for n in ("ct_projector", "parallel", "fan_equiangluar", "cone", "tomo")}
        mods["prior"] = importlib.import_module("ct_projector.prior.numpy.recon_prior")
        for m in mods.values():
            assert m.__file__.startswith(str(root))
        yield mods
    finally:
        sys.path.remove(str(root))
        for k in [k for k in sys.modules if k == "ct_projector" or k.startswith("ct_projector.")]:
            del sys.modules[k]


def _projector(ref, p):
    """The reference's ct_projector class with the case's geometry."""
    q = ref["ct_projector"].ct_projector()
    for k, v in p.as_dict().items():
        setattr(q, k, v.item() if hasattr(v, "item") and np.ndim(v) == 0 else v)
    return q


def test_library_is_ours(ref):
    assert ref["parallel"].module.ctpVersion  # an entry only libctp.so has
    assert ref["ct_projector"].set_device(0) == 0


@pytest.mark.parametrize("name", ["par_basic", "par_wide"])
def test_parallel_module(ref, name):
    from ctprojector_b200.projector.numpy import parallel as ours

    p, inp, golden = load_golden(name)
    q = _projector(ref, p)
    R = ref["parallel"]
    img, ang = inp["img"].astype(np.float32), inp["angles"].astype(np.float32)
    fp = R.distance_driven_fp(q, img, ang)
    assert np.array_equal(fp, ours.distance_driven_fp(p, img, ang))
    assert rel_l2(fp, golden["fp"]) <= TOL
    y = golden["fp"]
    assert rel_l2(R.distance_driven_bp(q, y, ang), golden["bp"]) <= TOL
    f = R.ramp_filter(q, y, "hann")
    assert np.array_equal(f, ours.ramp_filter(p, y, "hann"))
    assert rel_l2(f, golden["filter_hann"]) <= TOL
    assert rel_l2(R.distance_driven_bp(q, golden["filter_hann"], ang, True), golden["bp_fbp"]) <= TOL
    assert rel_l2(R.pixel_driven_bp(q, golden["filter_hann"], ang), golden["pixel_bp"]) <= TOL


@pytest.mark.parametrize("name", ["fan_basic", "fan_wide"])
def test_fan_module(ref, name):
    from ctprojector_b200.projector.numpy import fan_equiangluar as ours

    p, inp, golden = load_golden(name)
    q = _projector(ref, p)
    R = ref["fan_equiangluar"]
    img, ang = inp["img"].astype(np.float32), inp["angles"].astype(np.float32)
    fp = R.distance_driven_fp(q, img, ang)
    assert np.array_equal(fp, ours.distance_driven_fp(p, img, ang))
    assert rel_l2(fp, golden["fp"]) <= TOL
    y = golden["fp"]
    assert rel_l2(R.distance_driven_bp(q, y, ang), golden["bp"]) <= TOL
    assert rel_l2(R.ramp_filter(q, y, "hann"), golden["filter_hann"]) <= TOL
    assert rel_l2(R.distance_driven_bp(q, golden["filter_hann"], ang, True), golden["bp_fbp"]) <= TOL
    assert rel_l2(R.fbp_bp(q, golden["filter_hann"], ang), golden["fbp_bp"]) <= TOL
    # the fan Siddon pair: the reference's FP32 intrinsics put its own outputs
    # up to 6.4e-5 from exact rays (the GPU parity tests bound ours by 1e-5)
    assert rel_l2(R.siddon_fp(q, img, ang), golden["siddon_fp"]) <= 1e-4
    assert rel_l2(R.siddon_bp(q, golden["siddon_fp"], ang), golden["siddon_bp"]) <= 1e-4


def test_cone_module(ref):
    p, inp, golden = load_golden("siddon")
    q = _projector(ref, p)
    R = ref["cone"]
    geo = [inp[k].astype(np.float32) for k in ("det_center", "det_u", "det_v", "src")]
    fp = R.siddon_fp_arbitrary(q, inp["img"], *geo)
    assert rel_l2(fp, golden["fp"]) <= TOL
    assert rel_l2(R.siddon_bp_arbitrary(q, golden["fp"], *geo), golden["bp"]) <= TOL


def test_tomo_module(ref):
    p, inp, golden = load_golden("tomo")
    q = _projector(ref, p)
    R = ref["tomo"]
    dc, src = inp["det_center"].astype(np.float32), inp["src"].astype(np.float32)
    fp = R.distance_driven_fp(q, inp["img"], dc, src)
    assert rel_l2(fp, golden["fp"]) <= TOL
    # the reference back-projects item 0's weighted projections for every item
    bp = R.distance_driven_bp(q, golden["fp"], dc, src)
    assert rel_l2(bp[0], golden["bp"][0]) <= TOL


def test_prior_module(ref, oracle):
    rng = np.random.default_rng(5)
    img = rng.uniform(0, 1, (1, 6, 20, 24)).astype(np.float32)
    w = (0.5, 1.0, 2.0)
    s1, s2, var = ref["prior"].tv_sqs(img, w, 1e-6)
    o1, o2, _ = oracle.tv_sqs(img, w, 1e-6)
    assert rel_l2(s1, o1) <= TOL and rel_l2(s2, o2) <= TOL
