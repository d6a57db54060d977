"""The sequence driver's GPU kernels (csrc/imgproc.cu) against oracle/imgproc.py, bit-exact:
cv::pyrDown (evaluate.cc:176-178; the oracle is pinned against OpenCV on the CPU), depthUp
(evaluate.cc:121-135), the min/max depth mask (:278-289) and the colour view (:291-307)."""
import ctypes

import numpy as np
import pytest

from oracle import imgproc as oip

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("H,W,pad", [(480, 640, 0), (481, 641, 3), (2, 2, 0), (3, 5, 1), (1080, 1920, 0),
                                     (33, 17, 5)])
def test_pyr_down(pm_lib, H, W, pad):
    rng = np.random.default_rng(H + W)
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    src = torch.zeros((H, W + pad), dtype=torch.uint8, device="cuda")
    src[:, :W] = torch.from_numpy(img).cuda()
    dW, dH = W // 2, H // 2
    dst = torch.full((dH, dW + 2), 7, dtype=torch.uint8, device="cuda")
    assert pm_lib.pm_pyr_down_u8(W, H, vp(src), W + pad, vp(dst), dW + 2, stream()) == 0
    got = dst.cpu().numpy()
    np.testing.assert_array_equal(got[:, :dW], oip.pyr_down(img))
    assert (got[:, dW:] == 7).all()          # nothing written past the row


def test_pyr_down_rejects_tiny(pm_lib):
    t = torch.zeros(4, dtype=torch.uint8, device="cuda")
    assert pm_lib.pm_pyr_down_u8(1, 4, vp(t), 1, vp(t), 1, stream()) != 0


def test_depth_up_and_mask(pm_lib):
    rng = np.random.default_rng(4)
    H, W = 120, 160
    d = (rng.random((H, W)) * 25).astype(np.float32)
    d[rng.random(d.shape) < 0.1] = 1000.0
    src = torch.from_numpy(d).cuda()
    up = torch.empty((2 * H, 2 * W), dtype=torch.float32, device="cuda")
    assert pm_lib.pm_depth_up2(W, H, vp(src), 0, vp(up), 0, stream()) == 0
    np.testing.assert_array_equal(up.cpu().numpy(), oip.depth_up2(d))
    assert pm_lib.pm_depth_range_mask(2 * W, 2 * H, vp(up), 0, ctypes.c_float(0.2), ctypes.c_float(20.0),
                                      stream()) == 0
    np.testing.assert_array_equal(up.cpu().numpy(), oip.range_mask(oip.depth_up2(d), 0.2, 20.0))


@pytest.mark.parametrize("kind", ["masked", "constant", "nan", "wide"])
def test_colorize(pm_lib, kind):
    rng = np.random.default_rng(8)
    H, W = 240, 320
    d = (rng.random((H, W)) * 19.8 + 0.2).astype(np.float32)
    d[rng.random(d.shape) < 0.3] = 0
    if kind == "constant":
        d[:] = 2.5
    elif kind == "nan":
        d[5, 7] = np.nan
    elif kind == "wide":
        d = (rng.standard_normal((H, W)) * 1e3).astype(np.float32)
    src = torch.from_numpy(d).cuda()
    level = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    bgr = torch.empty((H, W, 3), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(2, dtype=torch.int32, device="cuda")
    assert pm_lib.pm_colorize_depth(W, H, vp(src), 0, vp(level), 0, vp(bgr), 0, vp(scratch), stream()) == 0
    wl, wb = oip.colorize(d)
    np.testing.assert_array_equal(level.cpu().numpy(), wl)
    np.testing.assert_array_equal(bgr.cpu().numpy(), wb)
