"""16-bit affine sinogram storage (ctp_quantize_u16, ctp_dequantize_u16,
ctp_ramp_filter_u16): the rounding bound of every sample, the in-place
residual, the filter that reads the codes against the exact filter of the
dequantized values, and ragged and constant views."""
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


def _sinogram(shape, seed):
    rng = np.random.default_rng(seed)
    y = rng.uniform(-0.05, 8.0, shape).astype(np.float32)
    return torch.tensor(y, device="cuda")


@pytest.mark.parametrize("shape", [(3, 17, 1, 129), (1, 5, 7, 33), (2, 1, 1, 1), (4, 360, 1, 736)])
def test_round_trip_within_half_a_step(shape):
    from ctprojector_b200 import quant

    y = _sinogram(shape, sum(shape))
    q = quant.quantize(y)
    assert q.code.dtype == torch.int16 and tuple(q.lo.shape) == shape[:2]
    back = quant.dequantize(q)
    torch.cuda.synchronize()
    yv = y.reshape(shape[0] * shape[1], -1)
    lo, hi = yv.min(1).values, yv.max(1).values
    assert torch.equal(q.lo.reshape(-1), lo)
    step = q.step.reshape(-1, 1)
    err = (back.reshape(yv.shape) - yv).abs()
    # half a step, plus the FP32 rounding of lo + step * code
    bound = step / 2 + 4 * torch.finfo(torch.float32).eps * yv.abs().max(1, keepdim=True).values
    assert bool(torch.all(err <= bound))
    # codes span the range: the minimum codes to 0 and the maximum to 65535
    codes = q.code.reshape(yv.shape).to(torch.int32) & 0xFFFF
    if shape[2] * shape[3] > 1:
        assert int(codes.min()) == 0 and int(codes.max()) == 65535
    # the host form of the stored values equals the device one to one FP32 rounding
    assert rel_l2(q.cpu().float().numpy(), back.cpu().numpy()) <= 1e-7


def test_constant_view_and_subtract():
    from ctprojector_b200 import quant

    y = _sinogram((2, 4, 1, 50), 3)
    y[1, 2] = 1.25  # a constant view: step 0, every code 0
    q = quant.quantize(y)
    back = quant.dequantize(q)
    torch.cuda.synchronize()
    assert float(q.step[1, 2]) == 0.0 and bool(torch.all(back[1, 2] == 1.25))
    r = torch.full_like(y, 3.0)
    quant.sub_dequantized_(r, q)
    torch.cuda.synchronize()
    assert torch.allclose(r, 3.0 - back, rtol=0, atol=1e-6)


@pytest.mark.parametrize("fan", [True, False])
def test_filter_reads_codes_like_dequantized_values(fan):
    """ctp_ramp_filter_u16 dequantizes with the same FP32 operation as
    ctp_dequantize_u16, so it equals the exact filter of those values."""
    from ctprojector_b200 import quant
    from ctprojector_b200.projector import _device as D
    from ctprojector_b200.projector.cupy.ct_projector import ct_projector

    p = ct_projector()
    p.nu, p.nv, p.du, p.dv, p.off_u, p.off_v, p.dsd, p.dso = 300, 2, 1.2858 if fan else 0.8, 1.0, 0.3, 0.0, 1085.6, 595.0
    y = _sinogram((3, 45, 2, 300), 7)
    q = quant.quantize(y)
    geom = 0 if fan else 1
    a = quant.ramp_filter(p, q, "hann", geom)
    b = D.ramp_filter(p, quant.dequantize(q), "hann", geom, exact=True)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    # and it is close to the filter of the unquantized sinogram
    c = D.ramp_filter(p, y, "hann", geom, exact=True)
    assert rel_l2(a.cpu().numpy(), c.cpu().numpy()) <= 1e-3


def test_filter_rejects_detectors_beyond_the_one_launch_filter():
    from ctprojector_b200._lib import CTP_ERR_UNSUPPORTED, Geometry, lib

    g = Geometry(1, 1, 1, 1, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 4000, 1, 2, 0.8, 1.0, 0.0, 0.0, 0.0, 0.0)
    t = torch.zeros(16, device="cuda")
    p = ctypes.c_void_p(t.data_ptr())
    assert lib().ctp_ramp_filter_u16(p, p, p, p, ctypes.byref(g), 1, 2, None) == CTP_ERR_UNSUPPORTED
