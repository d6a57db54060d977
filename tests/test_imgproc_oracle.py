"""The oracle of the sequence driver's image work (oracle/imgproc.py) pinned against OpenCV, the
library the reference calls (evaluate.cc:176-178 cv::pyrDown, :296 cv::normalize; the grey
conversion of cv::cvtColor), and the debug argmin against a literal transcription of
stereo_mapper.cpp:636-660 on the reference's own cost volume (tests/golden/ref_40x32x32.npz)."""
import os
from fractions import Fraction

import numpy as np
import pytest

from conftest import ROOT
from oracle import imgproc as ip

cv2 = pytest.importorskip("cv2")


@pytest.mark.parametrize("H,W", [(2, 2), (3, 5), (5, 3), (2, 9), (9, 2), (4, 4), (33, 17), (480, 640), (481, 641),
                                 (240, 376)])
def test_pyr_down_matches_opencv(H, W):
    rng = np.random.default_rng(H * 1000 + W)
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    ours = ip.pyr_down(img)
    ref = cv2.pyrDown(img, dstsize=(W // 2, H // 2))
    assert ours.shape == (H // 2, W // 2)
    np.testing.assert_array_equal(ours, ref)


def test_pyr_down_extremes():
    for v in (0, 255):
        img = np.full((16, 16), v, np.uint8)
        np.testing.assert_array_equal(ip.pyr_down(img), cv2.pyrDown(img, dstsize=(8, 8)))
    img = (np.indices((20, 30)).sum(0) % 2 * 255).astype(np.uint8)   # checkerboard: every sum is a .5 case
    np.testing.assert_array_equal(ip.pyr_down(img), cv2.pyrDown(img, dstsize=(15, 10)))


def test_fma_is_correctly_rounded():
    rng = np.random.default_rng(5)
    x = (rng.random(2000) * 40 - 5).astype(np.float32)
    a, b = np.float32(255.0 / 19.7), np.float32(-0.2 * 255.0 / 19.7)
    got = ip._fma_f32(x, a, b)
    for xi, gi in zip(x[:400], got[:400]):
        exact = Fraction(float(xi)) * Fraction(float(a)) + Fraction(float(b))
        # the two float32 neighbours of the exact value; got must be the nearer (ties to even)
        f = np.float32(float(exact))
        cands = [f, np.nextafter(f, np.float32(np.inf)), np.nextafter(f, np.float32(-np.inf))]
        best = min(cands, key=lambda c: (abs(Fraction(float(c)) - exact), int(np.float32(c).view(np.uint32)) & 1))
        assert gi == best


@pytest.mark.parametrize("seed", range(4))
def test_normalize_matches_opencv(seed):
    rng = np.random.default_rng(seed)
    d = (rng.random((240, 320)) * 19.8 + 0.2).astype(np.float32)
    d[rng.random(d.shape) < 0.3] = 0
    np.testing.assert_array_equal(ip.normalize_u8(d), cv2.normalize(d, None, 0, 255, cv2.NORM_MINMAX, cv2.CV_8U))


def test_normalize_ties_and_constant_map():
    d = np.arange(0, 11, dtype=np.float32)[None, :] * np.float32(0.5)
    np.testing.assert_array_equal(ip.normalize_u8(d), cv2.normalize(d, None, 0, 255, cv2.NORM_MINMAX, cv2.CV_8U))
    c = np.full((8, 8), 3.0, np.float32)
    np.testing.assert_array_equal(ip.normalize_u8(c), cv2.normalize(c, None, 0, 255, cv2.NORM_MINMAX, cv2.CV_8U))


def test_grey_matches_cvtcolor():
    rng = np.random.default_rng(9)
    rgb = rng.integers(0, 256, (200, 300, 3), dtype=np.uint8)
    np.testing.assert_array_equal(ip.rgb_to_grey(rgb[..., 0], rgb[..., 1], rgb[..., 2]),
                                  cv2.cvtColor(rgb, cv2.COLOR_RGB2GRAY))


def test_range_mask_and_depth_up():
    d = np.array([[0.1, 0.2, 5.0, 20.0, 20.5, np.float32(np.nan)]], np.float32)
    m = ip.range_mask(d, 0.2, 20.0)
    np.testing.assert_array_equal(m[0, :5], np.array([0, 0.2, 5.0, 20.0, 0], np.float32))
    assert np.isnan(m[0, 5])
    u = ip.depth_up2(np.arange(6, dtype=np.float32).reshape(2, 3))
    assert u.shape == (4, 6) and u[3, 5] == 5 and u[2, 1] == 3


def test_hue_ramp_is_continuous():
    lv = np.arange(256)
    c = ip.hue_ramp(lv[None, :])[0].astype(int)
    assert tuple(c[0]) == (0, 0, 255)          # B, G, R: red at level 0
    assert np.abs(np.diff(c, axis=0)).max() <= 5


def _case_loop(cost, D, dep_sample):
    """stereo_mapper.cpp:636-660 transcribed literally (double min, strict <)."""
    H, W, _ = cost.shape
    out = np.zeros((H, W), np.float32)
    for i in range(H):
        for j in range(W):
            mn, mi = 100000.0, None
            for d in range(D):
                if float(cost[i, j, d]) < mn:
                    mn, mi = float(cost[i, j, d]), d
            if mn < 1e-5:
                out[i, j] = 10000.0
            elif mi == 0 or mi == D - 1:
                out[i, j] = 0.0
            else:
                out[i, j] = np.float32(1.0) / (np.float32(mi) * np.float32(dep_sample))
    return out


@pytest.mark.parametrize("vol", ["A_cost", "A_sgm", "B_cost", "B_sgm"])
def test_case_argmin_matches_the_host_loop_on_reference_volumes(vol):
    z = np.load(os.path.join(ROOT, "tests", "golden", "ref_40x32x32.npz"))
    v = z[vol]
    ds = float(z["dep_sample"])
    dep, idx = ip.case_argmin(v, 0.0, ds)
    np.testing.assert_array_equal(dep, _case_loop(v, v.shape[2], ds))
    if vol.endswith("cost"):
        assert (dep == 10000.0).any()      # unmeasured voxels (-1) give the no-overlap value
