"""Host-side logic: the ct_projector class, config loading, plug-in dispatch,
error policy, filter names and the synthetic inputs."""
import numpy as np
import pytest


def test_defaults_match_reference():
    from ctprojector_b200.projector.numpy import ct_projector

    p = ct_projector()
    assert (p.nview, p.nu, p.nv, p.nx, p.ny, p.nz) == (720, 512, 512, 512, 512, 512)
    assert (p.dsd, p.dso, p.du, p.dv) == (1085.6, 595, 1.2, 1.2)


def test_from_file(tmp_path):
    from ctprojector_b200.projector.cupy import ct_projector

    cfg = tmp_path / "g.cfg"
    cfg.write_text("[geometry]\nnx=640\nny=640\nnz=1\ndx_mm=0.75\ndsd_mm=1086.5\nnview=2304\noff_u=-1.125\n")
    p = ct_projector()
    p.from_file(str(cfg))
    assert p.nx == 640 and isinstance(p.nx, int)
    assert p.nview == 2304 and isinstance(p.nview, int)
    assert p.dx == np.float32(0.75) and p.dsd == np.float32(1086.5)
    assert p.off_u == np.float32(-1.125)


def test_plugin_merges_default_kwargs():
    from ctprojector_b200.projector.numpy import ct_projector

    calls = []
    p = ct_projector()
    p.set_projector(lambda proj, img, **kw: calls.append(("fp", kw)) or img, angles=1, branchless=False)
    p.set_backprojector(lambda proj, prj, **kw: calls.append(("bp", kw)) or prj, angles=2)
    p.fp(0, branchless=True)
    p.bp(0)
    assert calls == [("fp", {"branchless": True, "angles": 1}), ("bp", {"angles": 2})]


def test_power_method_on_a_known_operator():
    from ctprojector_b200.projector.numpy import ct_projector

    p = ct_projector()
    p.nx, p.ny, p.nz = 4, 3, 1
    A = np.diag(np.arange(1, 13, dtype=np.float64))
    p.set_projector(lambda proj, x: (A @ x.reshape(-1)).reshape(x.shape))
    p.set_backprojector(lambda proj, y: (A.T @ y.reshape(-1)).reshape(y.shape))
    assert p.calc_projector_norm(niter=60) == pytest.approx(12.0, rel=1e-3)
    assert np.allclose(p.calc_norm_img().reshape(-1), np.arange(1, 13) ** 2)


def test_get_angles():
    from ctprojector_b200.projector.cupy import ct_projector

    p = ct_projector()
    p.nview = 8
    a = p.get_angles()
    assert a.dtype == np.float32 and np.allclose(a, np.arange(8) * np.pi / 4)


def test_filter_names():
    from ctprojector_b200.projector._device import filter_code

    assert [filter_code(s) for s in ("hamming", "HANN", "Cosine", "ramlak", "xyz")] == [1, 2, 3, 0, 0]


def test_strict_policy():
    from ctprojector_b200 import errors

    assert errors.is_strict()
    errors.set_strict(False, thread_local=True)
    assert not errors.is_strict()
    errors.set_strict(True, thread_local=True)
    assert errors.is_strict()


def test_phantom_statistics():
    from ctprojector_b200 import synthetic as S

    img = S.ellipse_phantom(np.random.default_rng(S.seed_for(2)), 128, 128, 0.8, 0.8)
    assert img.dtype == np.float32 and img.shape == (128, 128)
    inside = img[img > 0]
    assert 0.009 < np.percentile(inside, 10) and inside.max() < 0.031  # partial pixels only at edges
    r = 0.45 * 128 * 0.8
    assert abs((img > 0).mean() - np.pi * r * r / (128 * 0.8) ** 2) < 0.02


def test_poisson_log_is_seeded():
    from ctprojector_b200 import synthetic as S

    prj = np.full((2, 3), 1.5, np.float32)
    a = S.poisson_log(prj, 1e5, np.random.default_rng(5))
    b = S.poisson_log(prj, 1e5, np.random.default_rng(5))
    assert np.array_equal(a, b) and abs(a.mean() - 1.5) < 0.05


def test_helical_geometry_is_orthonormal():
    from ctprojector_b200 import synthetic as S

    dc, du, dv, src = S.helical(16, 2.0, 595.0, 1085.6, 35.08)
    assert np.allclose(np.linalg.norm(du, axis=1), 1) and np.allclose((du * dv).sum(1), 0)
    assert np.allclose(np.linalg.norm(src[:, :2] - dc[:, :2], axis=1), 1085.6, rtol=1e-5)
    assert np.allclose((du * (src - dc)).sum(1), 0, atol=1e-3)
