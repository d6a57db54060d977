"""StereoBatch: the batched form of the C ABI (pm_batch_*).

Many independent sequences, each with its own configuration, stepped together: every run() is
one keyframe of every sequence (initReference, the source updates, outputFusion), issued by the
library as one CUDA-graph launch.  This module only marshals pointers.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, load
from .mapper import _d


def _addr(x):
    return ctypes.c_void_p(x.data_ptr() if hasattr(x, "data_ptr") else x.ctypes.data)


class StereoBatch:
    """configs: list of dicts of pm_config fields, each with width, height and num_planes."""

    def __init__(self, configs, num_sources: int, lanes: int = 0, host_io: bool = True, autotune: bool = False,
                 priority: bool = False, persistent: bool = False, stats: bool = False):
        self.lib = load()
        n = len(configs)
        arr = (_lib.PmConfig * n)()
        self.shapes = []
        for i, c in enumerate(configs):
            c = dict(c)
            W, H, D = c.pop("width"), c.pop("height"), c.pop("num_planes")
            self.lib.pm_config_default(ctypes.byref(arr[i]), W, H, D)
            for k, v in c.items():
                if not hasattr(arr[i], k):
                    raise TypeError(f"unknown parameter {k}")
                setattr(arr[i], k, v)
            self.shapes.append((H, W))
        self.S = num_sources
        self.host_io = host_io
        flags = ((_lib.PM_BATCH_HOST_IO if host_io else 0) | (_lib.PM_BATCH_AUTOTUNE if autotune else 0) |
                 (_lib.PM_BATCH_PRIORITY if priority else 0) | (_lib.PM_BATCH_PERSISTENT if persistent else 0) |
                 (_lib.PM_BATCH_STATS if stats else 0))
        b = ctypes.c_void_p()
        check(self.lib.pm_batch_create(arr, n, num_sources, lanes, flags, ctypes.byref(b)), None, "pm_batch_create")
        self.b = b
        self.n = n

    def close(self):
        if getattr(self, "b", None):
            self.lib.pm_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != 0:
            msg = self.lib.pm_batch_last_error(self.b)
            raise _lib.PmError(st, f"{what}: {msg.decode() if msg else ''}")

    def init_intrinsic(self, seq: int, K, dep_sample: float):
        k, kp = _d(K)
        self._check(self.lib.pm_batch_init_intrinsic(self.b, seq, kp, float(dep_sample)), "pm_batch_init_intrinsic")

    def frame_ptr(self, seq: int, frame: int) -> int:
        p = ctypes.c_void_p()
        self._check(self.lib.pm_batch_frame(self.b, seq, frame, ctypes.byref(p)), "pm_batch_frame")
        return p.value

    def set_frame(self, seq: int, frame: int, img):
        """Copies a uint8 HxW image (numpy array or contiguous torch tensor, host or CUDA) into
        the next step's frame buffer."""
        H, W = self.shapes[seq]
        if not hasattr(img, "data_ptr"):
            img = np.ascontiguousarray(img, np.uint8)
        assert tuple(img.shape) == (H, W)
        self._check(self.lib.pm_batch_put_frame(self.b, seq, frame, _addr(img), W), "pm_batch_put_frame")

    def set_poses(self, seq: int, R_ref, T_ref, R_src, T_src):
        r, rp = _d(R_ref)
        t, tp = _d(T_ref)
        rs, rsp = _d(np.stack([np.asarray(R, np.float64).reshape(9) for R in R_src]))
        ts, tsp = _d(np.stack([np.asarray(T, np.float64).reshape(3) for T in T_src]))
        self._check(self.lib.pm_batch_set_poses(self.b, seq, rp, tp, rsp, tsp), "pm_batch_set_poses")

    def run(self):
        self._check(self.lib.pm_batch_run(self.b), "pm_batch_run")

    def synchronize(self):
        self._check(self.lib.pm_batch_synchronize(self.b), "pm_batch_synchronize")

    def output(self, seq: int):
        """(fused depth, variance) of the last step: numpy copies of the pinned host outputs
        (host I/O mode) or the device addresses."""
        d, v = ctypes.c_void_p(), ctypes.c_void_p()
        self._check(self.lib.pm_batch_output(self.b, seq, ctypes.byref(d), ctypes.byref(v)), "pm_batch_output")
        if not self.host_io:
            return d.value, v.value
        H, W = self.shapes[seq]
        n = W * H
        dep = np.ctypeslib.as_array((ctypes.c_float * n).from_address(d.value)).reshape(H, W).copy()
        var = np.ctypeslib.as_array((ctypes.c_float * n).from_address(v.value)).reshape(H, W).copy()
        return dep, var

    def copy_output(self, seq: int, depth=None, variance=None):
        """Fused depth and variance of the last step copied into numpy arrays or torch tensors
        (host or CUDA); new numpy arrays when not given."""
        H, W = self.shapes[seq]
        if depth is None:
            depth = np.empty((H, W), np.float32)
        if variance is None:
            variance = np.empty((H, W), np.float32)
        self._check(self.lib.pm_batch_copy_output(self.b, seq, _addr(depth), 0, _addr(variance), 0),
                    "pm_batch_copy_output")
        return depth, variance

    def wta_depth(self, seq: int, depth=None):
        """Winner-take-all depth of the last step (before fusion), copied into a numpy array or a
        torch tensor (host or CUDA); a new numpy array when not given."""
        H, W = self.shapes[seq]
        if depth is None:
            depth = np.empty((H, W), np.float32)
        self._check(self.lib.pm_batch_copy_wta_depth(self.b, seq, _addr(depth), 0), "pm_batch_copy_wta_depth")
        return depth

    def tuning(self, seq: int):
        w, s, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        self._check(self.lib.pm_batch_tuning(self.b, seq, ctypes.byref(w), ctypes.byref(s), ctypes.byref(ms)),
                    "pm_batch_tuning")
        return w.value, s.value, ms.value

    def stats(self, seq: int) -> dict:
        """pm_stats counters of sequence seq's last step (a batch made with stats=True)."""
        st = _lib.PmStats()
        self._check(self.lib.pm_batch_get_stats(self.b, seq, ctypes.byref(st)), "pm_batch_get_stats")
        return {n: int(getattr(st, n)) for n in _lib.STATS_FIELDS}

    def stream(self) -> int:
        return self.lib.pm_batch_stream(self.b)
