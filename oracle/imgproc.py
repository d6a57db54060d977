"""CPU restatement of the sequence driver's image work -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Only tests/ import this module, as the checker of the GPU kernels in
probabilistic_mapping_b200/csrc/imgproc.cu and of the debug argmin in csrc/sgm.cu.

* ``pyr_down``: cv::pyrDown(img, img, Size(W/2, H/2)) as evaluate.cc:176-178 and 221-225 call it
  (OpenCV's published Gaussian pyramid step, restated: 5x5 kernel [1 4 6 4 1]^T [1 4 6 4 1] / 256
  at even pixels, BORDER_REFLECT_101, (sum + 128) >> 8).  Pinned against cv2.pyrDown in
  tests/test_imgproc_oracle.py.
* ``depth_up2``: depthUp, evaluate.cc:121-135.
* ``range_mask``: evaluate.cc:278-289.
* ``normalize_u8``: cv::normalize(depth, 0, 255, NORM_MINMAX, CV_8U) of evaluate.cc:296, with the
  float conversion done as a single fused multiply-add; pinned against cv2.normalize.
* ``colorize``: the library's own hue ramp (csrc/imgproc.cu) and the black mask of
  evaluate.cc:298-306.
* ``rgb_to_grey``: BT.601 luma in 15-bit fixed point (the integer form of cv::cvtColor
  RGB2GRAY for 8-bit data); pinned against cv2.cvtColor.
* ``case_argmin``: the debug outputs of outputFusionCPU, stereo_mapper.cpp:628-662 (CASE 0, on
  the raw cost) and :672-706 (CASE 1, on the SGM sum).
"""
from __future__ import annotations

import numpy as np


def reflect101(p: np.ndarray, n: int) -> np.ndarray:
    """BORDER_REFLECT_101 of any integer offsets (iterated, as OpenCV's borderInterpolate)."""
    p = np.asarray(p, np.int64).copy()
    if n == 1:
        return np.zeros_like(p)
    while True:
        bad = (p < 0) | (p >= n)
        if not bad.any():
            return p
        p = np.where(p < 0, -p, np.where(p >= n, 2 * n - 2 - p, p))


_K5 = np.array([1, 4, 6, 4, 1], np.int64)


def pyr_down(img: np.ndarray) -> np.ndarray:
    """cv::pyrDown to (W/2, H/2) of a uint8 image (evaluate.cc:176-178)."""
    img = np.asarray(img, np.uint8)
    H, W = img.shape
    dH, dW = H // 2, W // 2
    ys = reflect101(2 * np.arange(dH)[:, None] + np.arange(-2, 3)[None, :], H)   # (dH, 5)
    xs = reflect101(2 * np.arange(dW)[:, None] + np.arange(-2, 3)[None, :], W)   # (dW, 5)
    src = img.astype(np.int64)
    rows = np.zeros((H, dW), np.int64)                 # horizontal pass on every source row
    for j in range(5):
        rows += _K5[j] * src[:, xs[:, j]]
    out = np.zeros((dH, dW), np.int64)
    for i in range(5):
        out += _K5[i] * rows[ys[:, i], :]
    return ((out + 128) >> 8).astype(np.uint8)


def depth_up2(d: np.ndarray) -> np.ndarray:
    """depthUp (evaluate.cc:121-135): every pixel repeated in a 2x2 block."""
    return np.repeat(np.repeat(np.asarray(d, np.float32), 2, axis=0), 2, axis=1)


def range_mask(d: np.ndarray, lo: float, hi: float) -> np.ndarray:
    """evaluate.cc:278-289: < lo -> 0, then > hi -> 0 (float32 comparisons)."""
    d = np.asarray(d, np.float32).copy()
    d[d < np.float32(lo)] = 0
    d[d > np.float32(hi)] = 0
    return d


def _fma_f32(x: np.ndarray, a: np.float32, b: np.float32) -> np.ndarray:
    """Correctly rounded float32 fma(x, a, b).  The product is exact in float64 and the float64
    sum s has the exact error e (TwoSum), so the true value is s + e.  Rounding s to float32
    already rounds s + e correctly unless s lies exactly halfway between two float32 values:
    float32 midpoints are float64 numbers, and |e| is below half a float64 step.  At a midpoint
    the sign of e picks the neighbour."""
    x = np.asarray(x, np.float32).astype(np.float64)
    p = x * np.float64(a)
    s = p + np.float64(b)
    bb = s - p
    e = (p - (s - bb)) + (np.float64(b) - bb)
    r = s.astype(np.float32)
    up = np.nextafter(r, np.float32(np.inf))
    dn = np.nextafter(r, np.float32(-np.inf))
    r64 = r.astype(np.float64)
    with np.errstate(invalid="ignore"):
        mid_above = s == (r64 + up.astype(np.float64)) / 2
        mid_below = s == (r64 + dn.astype(np.float64)) / 2
    r = np.where(mid_above & (e > 0), up, r)
    r = np.where(mid_below & (e < 0), dn, r)
    return r.astype(np.float32)


def normalize_u8(d: np.ndarray) -> np.ndarray:
    """cv::normalize(d, 0, 255, NORM_MINMAX, CV_8U) (evaluate.cc:296)."""
    d = np.asarray(d, np.float32)
    finite = d[~np.isnan(d)]
    smin = float(finite.min()) if finite.size else 0.0
    smax = float(finite.max()) if finite.size else 0.0
    rng = smax - smin
    scale = 255.0 / rng if rng > np.finfo(np.float64).eps else 0.0
    shift = 0.0 - smin * scale
    v = _fma_f32(d, np.float32(scale), np.float32(shift))
    v = np.where(np.isnan(v), np.float32(0), v)
    lv = np.rint(v.astype(np.float64))   # round half to even
    return np.clip(lv, 0, 255).astype(np.uint8)


def hue_ramp(level: np.ndarray) -> np.ndarray:
    """The library's colour map: (H, W) uint8 level -> (H, W, 3) B, G, R."""
    t = 5 * np.asarray(level, np.int64)
    k, f = t >> 8, t & 255
    r = np.select([k == 0, k == 1, k == 2, k == 3], [255, 255 - f, 0, 0], f)
    g = np.select([k == 0, k == 1, k == 2, k == 3], [f, 255, 255, 255 - f], 0)
    b = np.select([k == 0, k == 1, k == 2, k == 3], [0, 0, f, 255], 255)
    return np.stack([b, g, r], axis=-1).astype(np.uint8)


def colorize(d: np.ndarray):
    """The debug view of evaluate.cc:296-306 on an already range-masked map: (level, bgr)."""
    d = np.asarray(d, np.float32)
    level = normalize_u8(d)
    bgr = hue_ramp(level)
    bgr[d < np.float32(0.001)] = 0
    return level, bgr


def rgb_to_grey(r, g, b) -> np.ndarray:
    r, g, b = (np.asarray(v, np.int64) for v in (r, g, b))
    return ((9798 * r + 19235 * g + 3735 * b + 16384) >> 15).astype(np.uint8)


def case_argmin(vol: np.ndarray, rho0: float, drho: float) -> tuple[np.ndarray, np.ndarray]:
    """outputFusionCPU's CASE 0 / CASE 1 winner-take-all (stereo_mapper.cpp:636-660, 680-704)
    over an (H, W, D) float volume: the first plane holding a value below 100000 that no earlier
    plane undercuts; 10000 when that minimum is below FLOAT_EPS, 0 at the first and last plane,
    else 1 / fma(d, drho, rho0) in float32 (the reference has rho0 = 0, where the fused and the
    plain product agree).  Returns (depth, plane)."""
    vol = np.asarray(vol, np.float32)
    H, W, D = vol.shape
    v = np.where(np.isnan(vol), np.float32(np.inf), vol)
    v = np.where(v < np.float32(100000.0), v, np.float32(np.inf))
    idx = np.argmin(v, axis=2)                     # first occurrence of the minimum
    mn = np.take_along_axis(v, idx[..., None], 2)[..., 0]
    idx = np.where(np.isinf(mn), 0, idx)           # nothing below 100000: plane 0
    mn64 = np.where(np.isinf(mn), 100000.0, mn.astype(np.float64))
    rho = _fma_f32(idx.astype(np.float32), np.float32(drho), np.float32(rho0))   # one rounding
    with np.errstate(divide="ignore"):
        dep = (np.float32(1.0) / rho).astype(np.float32)
    dep = np.where((idx == 0) | (idx == D - 1), np.float32(0.0), dep)
    dep = np.where(mn64 < 1e-5, np.float32(10000.0), dep)
    return dep.astype(np.float32), idx.astype(np.int32)
