"""torch.autograd wrappers: FP and exact-adjoint BP as each other's backward,
finite-difference checks, and the checkpointed unrolled SQS-TV network."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _fan():
    from ctprojector_b200 import synthetic as S
    from ctprojector_b200.projector.cupy.ct_projector import ct_projector

    scan = S.Scan(48, 48, 1, 1.0, 1.0, 1.0, 72, 1, 1.2858, 1.0, 40)
    p = scan.projector(ct_projector)
    ang = torch.tensor(S.angles(40, 2 * np.pi), device="cuda")
    img = torch.tensor(S.ellipse_phantom(np.random.default_rng(5), 48, 48, 1.0, 1.0)[None, None], device="cuda")
    return p, ang, img


@pytest.mark.parametrize("geom", ["fan", "parallel"])
def test_fp_backward_is_exact_adjoint(geom):
    from ctprojector_b200 import autograd as AG
    from ctprojector_b200.projector import _device as D

    p, ang, img = _fan()
    x = img.clone().requires_grad_(True)
    y = AG.dd_fp(p, x, ang, geom)
    w = torch.rand_like(y)
    (y * w).sum().backward()
    ref = D.dd_bp(p, w, ang, 0 if geom == "fan" else 1, adjoint=True)
    assert torch.equal(x.grad, ref)


def test_bp_backward_is_forward():
    from ctprojector_b200 import autograd as AG
    from ctprojector_b200.projector import _device as D

    p, ang, img = _fan()
    prj = D.dd_fp(p, img, ang, 0)
    y = prj.clone().requires_grad_(True)
    x = AG.dd_bp(p, y, ang, "fan")
    w = torch.rand_like(x)
    (x * w).sum().backward()
    assert torch.equal(y.grad, D.dd_fp(p, w, ang, 0))


@pytest.mark.parametrize("geom", ["fan", "parallel"])
def test_least_squares_gradient_matches_finite_differences(geom):
    """L(x) = |Ax - b|^2 / 2 is quadratic, so central differences are exact
    up to rounding."""
    from ctprojector_b200 import autograd as AG

    p, ang, img = _fan()
    b = AG.dd_fp(p, img, ang, geom).detach()
    x = (img * 0.5).requires_grad_(True)
    loss = 0.5 * ((AG.dd_fp(p, x, ang, geom) - b) ** 2).sum()
    loss.backward()
    d = torch.randn_like(img)
    eps = 0.1
    with torch.no_grad():
        lp = 0.5 * ((AG.dd_fp(p, x + eps * d, ang, geom) - b).double() ** 2).sum()
        lm = 0.5 * ((AG.dd_fp(p, x - eps * d, ang, geom) - b).double() ** 2).sum()
    fd = float((lp - lm) / (2 * eps))
    an = float((x.grad.double() * d.double()).sum())
    assert abs(fd - an) <= 1e-3 * abs(an)


def test_siddon_autograd_pair():
    import cases

    from ctprojector_b200 import autograd as AG

    name, p, inp = cases.case_siddon()
    geo = [torch.tensor(inp[k], device="cuda") for k in ("det_center", "det_u", "det_v", "src")]
    x = torch.tensor(inp["img"], device="cuda").requires_grad_(True)
    y = AG.siddon_fp(p, x, *geo)
    w = torch.rand_like(y)
    (y * w).sum().backward()
    bp = AG.siddon_bp(p, w, *geo).detach()
    assert rel_l2(x.grad.cpu().numpy(), bp.cpu().numpy()) <= 1e-5
    # adjoint identity through the autograd pair
    lhs = float((y.detach().double() * w.double()).sum())
    rhs = float((x.detach().double() * bp.double()).sum())
    assert abs(lhs - rhs) / (y.detach().norm().item() * w.norm().item()) <= 1e-6


def test_tv_torch_matches_kernel():
    from ctprojector_b200.autograd import tv_sqs_torch
    from ctprojector_b200.prior import tv_sqs

    img = torch.rand(2, 4, 33, 29, device="cuda")
    for a, b in zip(tv_sqs_torch(img, (0.5, 1.0, 1.0)), tv_sqs(img, (0.5, 1.0, 1.0))):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) <= 1e-5


def test_unrolled_sqs_tv_checkpoint_and_training():
    from ctprojector_b200 import autograd as AG

    p, ang, img = _fan()
    fp = lambda x: AG.dd_fp(p, x, ang, "fan")  # noqa: E731
    bp = lambda y: AG.dd_bp(p, y, ang, "fan")  # noqa: E731
    with torch.no_grad():
        norm_img = bp(fp(torch.ones_like(img))).clamp_min(1e-6)
        y = fp(img)
    x0 = torch.zeros_like(img)
    grads = []
    for ckpt in (True, False):
        net = AG.UnrolledSQSTV(fp, bp, norm_img, n_iter=4, beta=1e-4, tv_weights=(0.0, 1.0, 1.0),
                               use_checkpoint=ckpt).cuda()
        out = net(x0, y)
        loss = ((out - img) ** 2).mean()
        loss.backward()
        grads.append(net.steps.grad.clone())
    assert rel_l2(grads[0].cpu().numpy(), grads[1].cpu().numpy()) <= 1e-5
    net = AG.UnrolledSQSTV(fp, bp, norm_img, n_iter=4, beta=1e-4, tv_weights=(0.0, 1.0, 1.0)).cuda()
    opt = torch.optim.Adam(net.parameters(), lr=0.05)
    losses = []
    for _ in range(20):
        opt.zero_grad()
        loss = ((net(x0, y) - img) ** 2).mean()
        loss.backward()
        opt.step()
        losses.append(float(loss))
    assert losses[-1] < losses[0]


def test_unrolled_cone_network_at_workload_size():
    """The differentiable cone workload: helical Siddon projector (1152 views
    over 2 turns, 736 x 64 panel) on a batch of 2 volumes of 64 x 512 x 512 at
    0.7 x 0.7 x 1.0 mm, driving a 4-iteration unrolled SQS-TV network with a
    learnable step per iteration and per-iteration checkpointing.  Checks the
    adjoint identity through autograd, a finite-difference directional
    derivative of a quadratic loss, and equal step gradients with and without
    checkpointing."""
    from ctprojector_b200 import autograd as AG
    from ctprojector_b200 import synthetic as S

    scan, (dc, du, dv, src), nb = S.config3()
    geo = [torch.tensor(a, device="cuda") for a in (dc, du, dv, src)]
    fp = lambda x: AG.siddon_fp(scan, x, *geo)  # noqa: E731
    bp = lambda y: AG.siddon_bp(scan, y, *geo)  # noqa: E731
    rng = np.random.default_rng(11)
    vol = torch.tensor(np.stack([S.ellipsoid_phantom(rng, 64, 512, 512, 1.0, 0.7, 0.7, supersample=1)
                                 for _ in range(nb)]), device="cuda")
    # adjoint identity through the autograd pair
    x = vol.clone().requires_grad_(True)
    y = fp(x)
    w = torch.rand_like(y)
    (y * w).sum().backward()
    lhs = float((y.detach().double() * w.double()).sum())
    rhs = float((vol.double() * x.grad.double()).sum())
    assert abs(lhs - rhs) / (y.detach().double().norm().item() * w.double().norm().item()) <= 1e-6
    # quadratic loss: central differences are exact up to rounding
    b = y.detach()
    x = (0.5 * vol).requires_grad_(True)
    (0.5 * ((fp(x) - b) ** 2).sum()).backward()
    d = torch.randn_like(vol) * (vol > 0)
    eps = 0.05
    with torch.no_grad():
        lp = 0.5 * ((fp(x + eps * d) - b).double() ** 2).sum()
        lm = 0.5 * ((fp(x - eps * d) - b).double() ** 2).sum()
    fd, an = float((lp - lm) / (2 * eps)), float((x.grad.double() * d.double()).sum())
    assert abs(fd - an) <= 1e-3 * abs(an)
    # the unrolled network, checkpointed and not
    with torch.no_grad():
        norm_img = bp(fp(torch.ones_like(vol[:1]))).clamp_min(1e-6)
    x0 = torch.zeros_like(vol)
    grads, outs = [], []
    for ckpt in (True, False):
        net = AG.UnrolledSQSTV(fp, bp, norm_img, n_iter=4, beta=1e-4, tv_weights=(1.0, 1.0, 1.0),
                               use_checkpoint=ckpt).cuda()
        out = net(x0, b)
        ((out - vol) ** 2).mean().backward()
        grads.append(net.steps.grad.clone())
        outs.append(out.detach())
        del net, out
    assert rel_l2(outs[0].cpu().numpy(), outs[1].cpu().numpy()) <= 1e-5
    assert rel_l2(grads[0].cpu().numpy(), grads[1].cpu().numpy()) <= 1e-4
    assert torch.all(torch.isfinite(grads[0])) and grads[0].abs().sum() > 0
