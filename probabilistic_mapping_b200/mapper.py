"""StereoMapper: the Python face of the drop-in C ABI.

Mirrors motion_stereo/stereo_mapper.h:26-63 method for method (initIntrinsic, initReference,
update, output, outputFusion) over numpy host arrays or torch CUDA tensors.  All work runs in
libpm_stereo.so; this module only marshals pointers.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PmBuffers, check, load


def _d(a):
    """(owner array, double*) for a 3x3 / 3-vector; keep the owner alive during the call."""
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    return a, ctypes.cast(a.ctypes.data, ctypes.POINTER(ctypes.c_double))


def _ptr(x):
    """Address of a numpy array or a torch tensor (host or CUDA)."""
    if hasattr(x, "data_ptr"):
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(x.ctypes.data)


class StereoMapper:
    """Drop-in counterpart of the reference's StereoMapper (stereo_mapper.cpp:27-244)."""

    def __init__(self, width: int, height: int, num_planes: int = 64, **params):
        self.lib = load()
        cfg = _lib.default_config(width, height, num_planes)
        for k, v in params.items():
            if not hasattr(cfg, k):
                raise TypeError(f"unknown parameter {k}")
            setattr(cfg, k, v)
        self.cfg = cfg
        h = ctypes.c_void_p()
        check(self.lib.pm_create(ctypes.byref(cfg), ctypes.byref(h)), None, "pm_create")
        self.h = h
        self.W, self.H, self.D = width, height, num_planes

    def close(self):
        if getattr(self, "h", None):
            self.lib.pm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st, what):
        check(st, self.h, what)

    def set_stream(self, stream_handle: int):
        self._check(self.lib.pm_set_stream(self.h, ctypes.c_void_p(stream_handle)), "pm_set_stream")

    # -- StereoMapper::initIntrinsic (stereo_mapper.cpp:51-61)
    def initIntrinsic(self, K, bf: float, dep_sample: float):
        k, kp = _d(K)
        self._check(self.lib.pm_init_intrinsic(self.h, kp, float(bf), float(dep_sample)), "initIntrinsic")

    # -- StereoMapper::initReference (stereo_mapper.cpp:63-71)
    def initReference(self, img, pitch: int = 0):
        img = self._img(img)
        self._check(self.lib.pm_init_reference(self.h, _ptr(img), pitch), "initReference")

    # -- StereoMapper::update (stereo_mapper.cpp:73-91)
    def update(self, img, R_l, T_l, R_r, T_r, pitch: int = 0):
        img = self._img(img)
        keep = [_d(x) for x in (R_l, T_l, R_r, T_r)]
        self._check(self.lib.pm_update(self.h, _ptr(img), pitch, *[p for _, p in keep]), "update")

    # -- StereoMapper::output (stereo_mapper.cpp:93-109)
    def output(self, out=None):
        if out is None:
            out = np.empty((self.H, self.W), np.float32)
        self._check(self.lib.pm_output(self.h, _ptr(out), 0), "output")
        return out

    # -- StereoMapper::outputFusion (stereo_mapper.cpp:111-244)
    def outputFusion(self, R, t, fx, fy, cx, cy, out=None, variance=None, want_variance=True):
        if out is None:
            out = np.empty((self.H, self.W), np.float32)
        if variance is None and want_variance:
            variance = np.empty((self.H, self.W), np.float32)
        r, rp = _d(R)
        tt, tp = _d(t)
        vp = _ptr(variance) if variance is not None else ctypes.c_void_p(0)
        self._check(self.lib.pm_output_fusion(self.h, _ptr(out), 0, vp, 0, rp, tp, float(fx), float(fy),
                                              float(cx), float(cy)), "outputFusion")
        return out, variance

    # -- outputFusionCPU's CASE 0 / 1 / 2 debug outputs (stereo_mapper.cpp:628-719)
    def outputCase(self, case: int, out=None):
        if out is None:
            out = np.empty((self.H, self.W), np.float32)
        self._check(self.lib.pm_output_case(self.h, int(case), _ptr(out), 0), "pm_output_case")
        return out

    def wta_depth(self, out=None):
        if out is None:
            out = np.empty((self.H, self.W), np.float32)
        self._check(self.lib.pm_get_wta_depth(self.h, _ptr(out), 0), "pm_get_wta_depth")
        return out

    def wta_index(self, out=None):
        if out is None:
            out = np.empty((self.H, self.W), np.int32)
        self._check(self.lib.pm_get_wta_index(self.h, _ptr(out)), "pm_get_wta_index")
        return out

    def get_state(self):
        arrs = [np.empty(self.W * self.H, np.float32) for _ in range(4)]
        self._check(self.lib.pm_get_state(self.h, *[_ptr(a) for a in arrs]), "pm_get_state")
        return arrs

    def set_state(self, alpha, beta, mu, sigma, R, t):
        arrs = [np.ascontiguousarray(a, np.float32).reshape(-1) for a in (alpha, beta, mu, sigma)]
        r, rp = _d(R)
        tt, tp = _d(t)
        self._check(self.lib.pm_set_state(self.h, *[_ptr(a) for a in arrs], rp, tp), "pm_set_state")

    def buffers(self) -> PmBuffers:
        b = PmBuffers()
        self._check(self.lib.pm_get_buffers(self.h, ctypes.byref(b)), "pm_get_buffers")
        return b

    def store_sgm(self, enable=True):
        self._check(self.lib.pm_debug_store_sgm(self.h, int(enable)), "pm_debug_store_sgm")

    def homography(self, i: int) -> np.ndarray:
        out = np.empty(12, np.float32)
        self._check(self.lib.pm_get_homography(self.h, i, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                    "pm_get_homography")
        return out

    def enable_stage_timing(self, enable=True):
        self._check(self.lib.pm_enable_stage_timing(self.h, int(enable)), "pm_enable_stage_timing")

    def stage_times(self) -> np.ndarray:
        """Milliseconds of [cost, sgm+wta, fusion, copy-out, cost kernel alone] of the last output call
        (the last entry is the cost stage without the FP16 form's rebase pass)."""
        out = np.zeros(5, np.float32)
        self._check(self.lib.pm_get_stage_times(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 5),
                    "pm_get_stage_times")
        return out

    def enable_stats(self, enable=True):
        self._check(self.lib.pm_enable_stats(self.h, int(enable)), "pm_enable_stats")

    def stats(self) -> dict:
        """Pixel counters of the last output call (pm_stats) as a dict of ints."""
        st = _lib.PmStats()
        self._check(self.lib.pm_get_stats(self.h, ctypes.byref(st)), "pm_get_stats")
        return {n: int(getattr(st, n)) for n in _lib.STATS_FIELDS}

    def synchronize(self):
        self._check(self.lib.pm_synchronize(self.h), "pm_synchronize")

    def _img(self, img):
        if hasattr(img, "data_ptr"):
            assert img.dtype.itemsize == 1 and img.is_contiguous() and tuple(img.shape) == (self.H, self.W)
            return img
        img = np.ascontiguousarray(img, np.uint8)
        if img.shape != (self.H, self.W):
            raise ValueError(f"image shape {img.shape} != {(self.H, self.W)}")
        return img
