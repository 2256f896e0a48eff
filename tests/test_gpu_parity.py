"""Parity of the sm_100a kernels (through the C ABI) with the FP64 oracle and
with the reference's own outputs (golden fixtures), on the seeded cases.

Tolerance: relative L2 <= 1e-5 in FP32 for every operator (the projector
parity bar); adjoint identity |<Ax,y> - <x,A^T y>| / (|Ax| |y|) <= 1e-6.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5
ADJ_TOL = 1e-6

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")


def host(t):
    torch.cuda.synchronize()
    return t.detach().float().cpu().numpy()


def mods(fan):
    from ctprojector_b200.projector.cupy import fan_equiangular, parallel

    return fan_equiangular if fan else parallel


DD_CASES = ["fan_basic", "fan_offsets", "par_basic", "par_offsets"]


def _case(name):
    import cases

    for fn in cases.ALL:
        n, p, inp = fn()
        if n == name:
            return p, inp
    raise KeyError(name)


@pytest.mark.parametrize("name", DD_CASES)
def test_dd_fp_matches_oracle(name, oracle):
    p, inp = _case(name)
    fan = name.startswith("fan")
    M = mods(fan)
    prj = host(M.distance_driven_fp(p, dev(inp["img"]), dev(inp["angles"])))
    ref = oracle.dd_fp(p, inp["img"], inp["angles"], "fan" if fan else "parallel")
    assert prj.shape == ref.shape
    assert rel_l2(prj, ref) <= TOL


@pytest.mark.parametrize("name", ["par_offsets", "par_wide", "fan_wide"])
def test_streamed_fp_stack_matches_oracle(name, oracle):
    """Stacks of 8 or more slices run the streamed forward projector (line
    tables copied into shared memory); parallel beams there sum each edge's
    running integrals over the lines and take the cell differences once."""
    p, inp = _case(name)
    fan = name.startswith("fan")
    rng = np.random.default_rng(11)
    base = inp["img"]
    reps = -(-8 // (base.shape[0] * base.shape[1]))
    img = np.concatenate([base * np.float32(1 + 0.25 * k) + rng.uniform(0, 0.2, base.shape).astype(np.float32)
                          for k in range(reps)]).astype(np.float32)
    assert img.shape[0] * img.shape[1] >= 8
    prj = host(mods(fan).distance_driven_fp(p, dev(img), dev(inp["angles"])))
    ref = oracle.dd_fp(p, img, inp["angles"], "fan" if fan else "parallel")
    assert rel_l2(prj, ref) <= TOL


@pytest.mark.parametrize("nu", [2300, 3000])
def test_fan_fp_wide_detector_matches_oracle(nu, oracle):
    """Fan detectors of more than 64 groups of 31 cells take one view per
    CTA with 12 (2300 cells) or 16 (3000 cells) edge groups per warp."""
    from cases import Proj

    p = Proj(nx=256, ny=256, nz=1, dx=1.0, dy=1.0, nu=nu, nv=1, du=0.4, dv=1.0, off_u=0.3, nview=40)
    rng = np.random.default_rng(nu)
    img = rng.uniform(0, 1, (2, 1, 256, 256)).astype(np.float32)
    ang = (np.arange(40) * 2 * np.pi / 40 + 0.05).astype(np.float32)
    prj = host(mods(True).distance_driven_fp(p, dev(img), dev(ang)))
    assert rel_l2(prj, oracle.dd_fp(p, img, ang, "fan")) <= TOL


@pytest.mark.parametrize("name", DD_CASES)
@pytest.mark.parametrize("is_fbp", [False, True])
def test_dd_bp_parity_matches_oracle(name, is_fbp, oracle):
    p, inp = _case(name)
    fan = name.startswith("fan")
    M = mods(fan)
    geom = "fan" if fan else "parallel"
    prj = oracle.dd_fp(p, inp["img"], inp["angles"], geom)
    img = host(M.distance_driven_bp(p, dev(prj), dev(inp["angles"]), is_fbp))
    ref = oracle.dd_bp(p, prj, inp["angles"], geom, is_fbp=is_fbp)
    assert rel_l2(img, ref) <= TOL


@pytest.mark.parametrize("name", DD_CASES)
def test_dd_bp_adjoint_matches_oracle(name, oracle):
    p, inp = _case(name)
    fan = name.startswith("fan")
    M = mods(fan)
    geom = "fan" if fan else "parallel"
    prj = oracle.dd_fp(p, inp["img"], inp["angles"], geom)
    img = host(M.distance_driven_bp(p, dev(prj), dev(inp["angles"]), adjoint=True))
    ref = oracle.dd_bp(p, prj, inp["angles"], geom, adjoint=True)
    assert rel_l2(img, ref) <= TOL


@pytest.mark.parametrize("name", DD_CASES)
def test_dd_adjoint_identity(name):
    p, inp = _case(name)
    fan = name.startswith("fan")
    M = mods(fan)
    rng = np.random.default_rng(7)
    x = inp["img"]
    ang = dev(inp["angles"])
    Ax = host(M.distance_driven_fp(p, dev(x), ang)).astype(np.float64)
    y = rng.uniform(0, 1, Ax.shape)
    Aty = host(M.distance_driven_bp(p, dev(y), ang, adjoint=True)).astype(np.float64)
    lhs, rhs = (Ax * y).sum(), (x.astype(np.float64) * Aty).sum()
    assert abs(lhs - rhs) / (np.linalg.norm(Ax) * np.linalg.norm(y)) <= ADJ_TOL


# The default filter replays the reference's FP32 construction of the windowed
# ramp (length 2nu-1 transforms); its distance to the exact FP64 filter is the
# reference's own rounding, up to REF_FILTER_TOL on these cases.  The exact
# mode (FP64 kernel, FP64 arithmetic) meets EXACT_FILTER_TOL against the oracle.
REF_FILTER_TOL = 1e-4
EXACT_FILTER_TOL = 1e-6


@pytest.mark.parametrize("name", DD_CASES + ["par_wide", "fan_wide"])
@pytest.mark.parametrize("ftype", ["hann", "hamming", "cosine", "ramlak"])
def test_ramp_filter_matches_oracle(name, ftype, oracle):
    p, inp = _case(name)
    fan = name.startswith("fan")
    M = mods(fan)
    geom = "fan" if fan else "parallel"
    # the same FP32 input on both sides (the filter magnifies input rounding)
    prj = oracle.dd_fp(p, inp["img"], inp["angles"], geom).astype(np.float32)
    ref = oracle.ramp_filter(p, prj, ftype, geom)
    assert rel_l2(host(M.ramp_filter(p, dev(prj), ftype, exact=True)), ref) <= EXACT_FILTER_TOL
    assert rel_l2(host(M.ramp_filter(p, dev(prj), ftype)), ref) <= REF_FILTER_TOL


@pytest.mark.parametrize("name", ["fan_basic", "fan_offsets"])
def test_fbp_bp_matches_oracle(name, oracle):
    from ctprojector_b200.projector.cupy import fan_equiangular as F

    p, inp = _case(name)
    prj = oracle.ramp_filter(p, oracle.dd_fp(p, inp["img"], inp["angles"], "fan"), "hann", "fan")
    img = host(F.fbp_bp(p, dev(prj), dev(inp["angles"])))
    ref = oracle.fbp_bp(p, prj, inp["angles"])
    assert rel_l2(img, ref) <= TOL


def test_siddon_matches_oracle(oracle):
    from ctprojector_b200.projector.cupy import cone

    p, inp = _case("siddon")
    a = [inp[k] for k in ("det_center", "det_u", "det_v", "src")]
    prj = host(cone.siddon_fp_arbitrary(p, dev(inp["img"]), *[dev(v) for v in a]))
    ref = oracle.siddon_fp(p, inp["img"], *a)
    assert rel_l2(prj, ref) <= TOL
    img = host(cone.siddon_bp_arbitrary(p, dev(ref), *[dev(v) for v in a]))
    ref_bp = oracle.siddon_bp(p, ref, *a)
    assert rel_l2(img, ref_bp) <= TOL


def test_siddon_full_size_volume_matches_oracle(oracle):
    """The 64 x 512 x 512 helical cone volume (0.7 x 0.7 x 1.0 mm, 736 x 64
    panel) with every 10th of its 360 views: rays cross ~700 voxels, where
    an FP32 alpha recurrence drifts (the reference's kernels differ from the
    FP64 oracle by 1.3e-5 (FP) and 5e-4 (BP) here); the anchored walk stays
    within the projector bar."""
    from cases import Proj

    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.projector.cupy import cone

    p = Proj(nx=512, ny=512, nz=64, dx=0.7, dy=0.7, dz=1.0, nu=736, nv=64, du=1.2858, dv=1.0, nview=36)
    geo = [np.ascontiguousarray(a[::10]) for a in S.helical(360, 1.0, 595.0, 1085.6, 64 * 595.0 / 1085.6)]
    img = S.ellipsoid_phantom(np.random.default_rng(0), 64, 512, 512, 1.0, 0.7, 0.7, supersample=1)[None]
    prj = host(cone.siddon_fp_arbitrary(p, dev(img), *[dev(a) for a in geo]))
    assert rel_l2(prj, oracle.siddon_fp(p, img, *geo)) <= TOL
    bp = host(cone.siddon_bp_arbitrary(p, dev(prj), *[dev(a) for a in geo]))
    assert rel_l2(bp, oracle.siddon_bp(p, prj, *geo)) <= TOL


def test_siddon_adjoint_identity():
    from ctprojector_b200.projector.cupy import cone

    p, inp = _case("siddon")
    a = [dev(inp[k]) for k in ("det_center", "det_u", "det_v", "src")]
    x = inp["img"].astype(np.float64)
    Ax = host(cone.siddon_fp_arbitrary(p, dev(x), *a)).astype(np.float64)
    y = np.random.default_rng(3).uniform(0, 1, Ax.shape)
    Aty = host(cone.siddon_bp_arbitrary(p, dev(y), *a)).astype(np.float64)
    assert abs((Ax * y).sum() - (x * Aty).sum()) / (np.linalg.norm(Ax) * np.linalg.norm(y)) <= ADJ_TOL


def test_tomo_matches_oracle(oracle):
    from ctprojector_b200.projector.cupy import tomo

    p, inp = _case("tomo")
    prj = host(tomo.distance_driven_fp(p, dev(inp["img"]), dev(inp["det_center"]), dev(inp["src"])))
    ref = oracle.tomo_fp(p, inp["img"], inp["det_center"], inp["src"])
    assert rel_l2(prj, ref) <= TOL
    img = host(tomo.distance_driven_bp(p, dev(ref), dev(inp["det_center"]), dev(inp["src"])))
    ref_bp = oracle.tomo_bp(p, ref, inp["det_center"], inp["src"])
    assert rel_l2(img, ref_bp) <= TOL


@pytest.mark.parametrize("cell", [0.1, 0.25, 0.5, 1.3])
def test_tomo_footprint_sizes_match_oracle(oracle, cell):
    """Detector cells of 0.1 to 1.3 mm under 0.4 mm voxels: the forward
    projector's footprints span up to 2 x 2 pixels per plane (straight-line
    path) or more (general loop), the back projector's up to 2 x 2, 3 x 3 or
    more cells per view; every path against the FP64 oracle."""
    from cases import Proj

    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.projector.cupy import tomo

    n = int(round(64 * 0.25 / cell))
    p = Proj(nx=96, ny=64, nz=10, dx=0.4, dy=0.4, dz=1.0, nu=2 * n, nv=n, du=cell, dv=cell, nview=9)
    dc, sr = S.tomo_geometry(9, 30.0, 650.0, -12.0)
    rng = np.random.default_rng(int(cell * 100))
    img = S.ellipsoid_phantom(rng, 10, 64, 96, 1.0, 0.4, 0.4, supersample=1)[None]
    prj = host(tomo.distance_driven_fp(p, dev(img), dev(dc), dev(sr)))
    ref = oracle.tomo_fp(p, img, dc, sr)
    assert rel_l2(prj, ref) <= TOL
    bp = host(tomo.distance_driven_bp(p, dev(ref), dev(dc), dev(sr)))
    assert rel_l2(bp, oracle.tomo_bp(p, ref, dc, sr)) <= TOL


# ----------------------------------------------------------------- vs the reference itself
@pytest.mark.parametrize("name", DD_CASES + ["kat", "par_wide", "fan_wide", "fan_45"])
def test_dd_matches_reference_golden(name):
    p, inp, ref = load_golden(name)
    fan = name.startswith("fan")
    M = mods(fan)
    ang = dev(inp["angles"])
    prj = host(M.distance_driven_fp(p, dev(inp["img"]), ang))
    assert rel_l2(prj, ref["fp"]) <= TOL
    if "bp" in ref:
        assert rel_l2(host(M.distance_driven_bp(p, dev(ref["fp"]), ang)), ref["bp"]) <= TOL
    src = ref.get("filter_hann", inp.get("prj"))
    assert rel_l2(host(M.distance_driven_bp(p, dev(src), ang, True)), ref["bp_fbp"]) <= TOL
    for f in ("hann", "hamming", "cosine", "ramlak"):
        if f"filter_{f}" in ref:
            assert rel_l2(host(M.ramp_filter(p, dev(ref["fp"]), f)), ref[f"filter_{f}"]) <= TOL
    if "fbp_bp" in ref:
        assert rel_l2(host(M.fbp_bp(p, dev(ref["filter_hann"]), ang)), ref["fbp_bp"]) <= TOL


def test_siddon_matches_reference_golden():
    from ctprojector_b200.projector.cupy import cone

    p, inp, ref = load_golden("siddon")
    a = [dev(inp[k]) for k in ("det_center", "det_u", "det_v", "src")]
    assert rel_l2(host(cone.siddon_fp_arbitrary(p, dev(inp["img"]), *a)), ref["fp"]) <= TOL
    assert rel_l2(host(cone.siddon_bp_arbitrary(p, dev(ref["fp"]), *a)), ref["bp"]) <= TOL


def test_tomo_matches_reference_golden():
    from ctprojector_b200.projector.cupy import tomo

    p, inp, ref = load_golden("tomo")
    dc, sr = dev(inp["det_center"]), dev(inp["src"])
    assert rel_l2(host(tomo.distance_driven_fp(p, dev(inp["img"]), dc, sr)), ref["fp"]) <= TOL
    # the reference back-projects batch item 0's weighted projections for every
    # item (distanceDriven3DBoxInt.cu:257-259); item 0 is comparable
    bp = host(tomo.distance_driven_bp(p, dev(ref["fp"]), dc, sr))
    assert rel_l2(bp[0], ref["bp"][0]) <= TOL


TOMO_FILTERS = (("hann", "hann", 1.0, 1.0), ("hamming_cut", "hamming", 0.8, 0.6), ("ramlak", "ramlak", 1.0, 1.0))


@pytest.mark.parametrize("key,name,cx,cz", TOMO_FILTERS)
def test_tomo_filter_matches_oracle_and_reference(oracle, key, name, cx, cz):
    """Tomosynthesis FBP filter: within the FP32 kernel construction of the
    FP64 oracle (1e-4, as the other reference-construction filters), and
    within 1e-5 of the reference's own output when the fixture holds it."""
    from ctprojector_b200.projector.cupy import tomo

    p, inp = _case("tomo")
    rng = np.random.default_rng(5)
    prj = rng.uniform(0, 1, (2, 9, p.nv, p.nu)).astype(np.float32)
    out = host(tomo.filter_fbp(p, dev(prj), dev(inp["det_center"]), dev(inp["src"]), name, cx, cz))
    assert rel_l2(out, oracle.tomo_filter(p, prj, inp["det_center"], inp["src"], name, cx, cz)) <= 1e-4
    _, ginp, ref = load_golden("tomo")
    if f"filter_{key}" in ref:
        # the reference filters every view with the first view's kernel
        out = host(tomo.filter_fbp(p, dev(ref["fp"]), dev(ginp["det_center"]), dev(ginp["src"]), name, cx, cz,
                                   first_view_kernel=True))
        assert rel_l2(out, ref[f"filter_{key}"]) <= TOL


@pytest.mark.parametrize("name", ["fan_basic", "fan_offsets", "fan_wide"])
def test_siddon_fan_matches_oracle_and_reference(oracle, name):
    """Fan-beam Siddon pair (numpy-module projector of the reference): CUDA
    vs the FP64 oracle and vs the reference's own outputs, and the adjoint
    identity."""
    from ctprojector_b200.projector.cupy import fan_equiangular as F
    from ctprojector_b200.projector.numpy import fan_equiangluar as NF

    p, inp = _case(name)
    ang = dev(inp["angles"])
    prj = host(F.siddon_fp(p, dev(inp["img"]), ang))
    assert rel_l2(prj, oracle.siddon_fan_fp(p, inp["img"], inp["angles"])) <= TOL
    bp = host(F.siddon_bp(p, dev(prj), ang))
    assert rel_l2(bp, oracle.siddon_fan_bp(p, prj, inp["angles"])) <= TOL
    assert rel_l2(NF.siddon_fp(p, inp["img"], inp["angles"]), prj) <= 1e-6  # host entry, same kernels
    rng = np.random.default_rng(2)
    y = rng.uniform(0, 1, prj.shape).astype(np.float32)
    aty = host(F.siddon_bp(p, dev(y), ang))
    assert abs(np.vdot(prj.astype(np.float64), y) - np.vdot(inp["img"].astype(np.float64), aty)) / (
        np.linalg.norm(prj) * np.linalg.norm(y)) <= ADJ_TOL
    _, ginp, ref = load_golden(name)
    if "siddon_fp" in ref:
        # the reference's FP32 intrinsic ray geometry and FP32 atomics: up to 6.4e-5 from the exact rays
        tol = 1e-4
        assert rel_l2(host(F.siddon_fp(p, dev(ginp["img"]), dev(ginp["angles"]))), ref["siddon_fp"]) <= tol
        assert rel_l2(host(F.siddon_bp(p, dev(ref["siddon_fp"]), dev(ginp["angles"]))), ref["siddon_bp"]) <= tol


@pytest.mark.parametrize("name", ["par_basic", "par_offsets", "par_wide"])
def test_pixel_driven_bp_matches_oracle_and_reference(oracle, name):
    from ctprojector_b200.projector.cupy import parallel as P
    from ctprojector_b200.projector.numpy import parallel as NP

    p, inp = _case(name)
    rng = np.random.default_rng(4)
    prj = rng.uniform(0, 1, (inp["img"].shape[0], len(inp["angles"]), p.nv, p.nu)).astype(np.float32)
    out = host(P.pixel_driven_bp(p, dev(prj), dev(inp["angles"])))
    assert rel_l2(out, oracle.pixel_bp_parallel(p, prj, inp["angles"])) <= TOL
    assert rel_l2(NP.pixel_driven_bp(p, prj, inp["angles"]), out) <= 1e-6
    _, ginp, ref = load_golden(name)
    if "pixel_bp" in ref:
        assert rel_l2(host(P.pixel_driven_bp(p, dev(ref["filter_hann"]), dev(ginp["angles"]))), ref["pixel_bp"]) <= TOL


@pytest.mark.parametrize("name", ["fan_wide", "par_wide", "fan_offsets"])
def test_host_module_exact_filter_matches_device(name, oracle):
    """The numpy modules' exact=True (host-array entry ctp_ramp_filter_host)
    runs the same one-launch FP64 filter as the device path."""
    from ctprojector_b200.projector.numpy import fan_equiangluar, parallel

    p, inp = _case(name)
    fan = name.startswith("fan")
    prj = oracle.dd_fp(p, inp["img"], inp["angles"], "fan" if fan else "parallel").astype(np.float32)
    a = (fan_equiangluar if fan else parallel).ramp_filter(p, prj, "hann", exact=True)
    b = host(mods(fan).ramp_filter(p, dev(prj), "hann", exact=True))
    assert np.array_equal(a, b)


BRANCHLESS_2D = ["fan_basic", "fan_offsets", "par_basic", "par_offsets", "par_wide", "fan_wide"]


@pytest.mark.parametrize("name", BRANCHLESS_2D)
def test_branchless_matches_reference_and_oracle(name, oracle):
    """branchless=True against the reference's branchless outputs
    (typeProjector bit 1) and the oracle's branchless mode: forward
    projection, normalised and FBP-weighted back projection."""
    p, inp, ref = load_golden(f"branchless_{name}")
    fan = name.startswith("fan")
    kind = "fan" if fan else "parallel"
    M = mods(fan)
    img, ang = inp["img"], inp["angles"]
    fp = host(M.distance_driven_fp(p, dev(img), dev(ang), True))
    assert rel_l2(fp, ref["fp"]) <= TOL
    assert rel_l2(fp, oracle.dd_fp(p, img, ang, kind, branchless=True)) <= TOL
    bp = host(M.distance_driven_bp(p, dev(ref["fp"]), dev(ang), False, True))
    assert rel_l2(bp, ref["bp"]) <= TOL
    assert rel_l2(bp, oracle.dd_bp(p, ref["fp"], ang, kind, branchless=True)) <= TOL
    bpf = host(M.distance_driven_bp(p, dev(ref["fp"]), dev(ang), True, True))
    assert rel_l2(bpf, ref["bp_fbp"]) <= TOL


def test_tomo_branchless_matches_reference():
    """The reference's branchless tomo tracer computes the box-integral
    operator: branchless=True gives its outputs (batch item 0; the back
    projection of view 0, which its pre-weight bug leaves intact)."""
    from ctprojector_b200.projector.cupy import tomo

    p, inp, ref = load_golden("branchless_tomo")
    dc, sr = dev(inp["det_center"]), dev(inp["src"])
    assert rel_l2(host(tomo.distance_driven_fp(p, dev(inp["img"]), dc, sr, True)), ref["fp"]) <= TOL
    bp = host(tomo.distance_driven_bp(p, dev(ref["fp"][:, :1]), dc[:1].contiguous(), sr[:1].contiguous(), True))
    assert rel_l2(bp, ref["bp_view0"]) <= TOL
