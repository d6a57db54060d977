"""CPU oracle for the motion-stereo path -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

A restatement of HKUST-Aerial-Robotics/probabilistic_mapping's motion_stereo kernels
(calc_cost.cu, sgm.cu, filter_cost.cu, depth_fusion.cu, convert.cu) and the StereoMapper
orchestration (stereo_mapper.cpp), compiled from oracle/pm_oracle.cpp.  Only tests/,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline / reference arm import this
module, and only as the checker or the timed CPU baseline.

``prec="f64"`` is the FP64 line-for-line transcription (the parity target); ``prec="f32"``
replays the B200 kernels' FP32 op order, for bit-exact comparisons.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libpm_oracle.so")
_lib = None

DEP_INF = 1000.0


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("W", ctypes.c_int), ("H", ctypes.c_int), ("D", ctypes.c_int),
        ("rho0", ctypes.c_double), ("drho", ctypes.c_double),
        ("intensity_scale", ctypes.c_double),
        ("cost_mode", ctypes.c_int), ("bilinear_quant", ctypes.c_int),
        ("num_paths", ctypes.c_int),
        ("p1", ctypes.c_double), ("p2", ctypes.c_double), ("tau_so", ctypes.c_double),
        ("q1", ctypes.c_double), ("q2", ctypes.c_double),
        ("var_scale", ctypes.c_double), ("uniqueness", ctypes.c_double),
        ("tree_compat", ctypes.c_int), ("sum_order", ctypes.c_int),
    ]


@dataclass
class Params:
    """Pipeline parameters; defaults are the reference's (parameters.cpp:12-18)."""
    W: int
    H: int
    D: int
    drho: float
    rho0: float = 0.0
    intensity_scale: float = 1.0
    cost_mode: int = 0          # 0 reference (bug-compatible), 1 corrected 3x3
    bilinear_quant: int = 0
    num_paths: int = 4
    p1: float = 8.0
    p2: float = 24.0
    tau_so: float = 4.0
    q1: float = 2.0
    q2: float = 3.0
    var_scale: float = 1.02
    uniqueness: float = 0.0
    tree_compat: int = 1
    sum_order: int = 1          # 0 reference path order, 1 grouped order of the B200 kernels

    def c(self) -> OrcParams:
        return OrcParams(self.W, self.H, self.D, self.rho0, self.drho, self.intensity_scale,
                         self.cost_mode, self.bilinear_quant, self.num_paths, self.p1, self.p2,
                         self.tau_so, self.q1, self.q2, self.var_scale, self.uniqueness,
                         self.tree_compat, self.sum_order)


def build(force: bool = False) -> str:
    """Compile oracle/pm_oracle.cpp (needs g++ with OpenMP)."""
    srcs = ("pm_oracle.cpp", "pm_oracle_diff.cpp", "pm_oracle.h")
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(os.path.join(_HERE, f)) for f in srcs)):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d, f, i32, u8, u32 = (P(ctypes.c_double), P(ctypes.c_float), P(ctypes.c_int32),
                              P(ctypes.c_uint8), P(ctypes.c_uint32))
        pp = P(OrcParams)
        L.orc_compose_homography.argtypes = [d, d, d, d, d, d]
        L.orc_relative_pose.argtypes = [d, d, d, d, d]
        L.orc_calc_cost_f64.argtypes = [pp, u8, u8, ctypes.c_int, d, d, d]
        L.orc_calc_cost_f32.argtypes = [pp, u8, u8, ctypes.c_int, d, f, f]
        L.orc_sgm_f64.argtypes = [pp, u8, d, d]
        L.orc_sgm_f32.argtypes = [pp, u8, f, f]
        L.orc_filter_f64.argtypes = [pp, d, d, i32]
        L.orc_filter_f32.argtypes = [pp, f, f, i32]
        L.orc_filter_classes_f32.argtypes = [pp, f, f, i32, u8]
        L.orc_tree_order.argtypes = [ctypes.c_int, ctypes.c_int, i32, i32]
        L.orc_fuse_gpu_f64.argtypes = [ctypes.c_int, ctypes.c_int, f, f] + [d] * 9 + [i32]
        L.orc_fuse_gpu_f32.argtypes = [ctypes.c_int, ctypes.c_int, f, f] + [f] * 9 + [i32]
        L.orc_fuse_gpu_counts_f32.argtypes = [ctypes.c_int, ctypes.c_int, f, f] + [f] * 9 + [i32, u32]
        L.orc_fuse_cpu.argtypes = [ctypes.c_int, ctypes.c_int, d, f, ctypes.c_int,
                                   f, f, f, f, f, u32]
        L.orc_fuse_cpu_counts.argtypes = [ctypes.c_int, ctypes.c_int, d, f, ctypes.c_int,
                                          f, f, f, f, f, u32, u32]
        L.orc_convert.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_uint64]
        dp = P(OrcDiffParams)
        L.orc_diff_forward.argtypes = [dp, d, d, d, d, d, d, d, u8]
        L.orc_diff_forward.restype = ctypes.c_double
        L.orc_diff_backward.argtypes = [dp, d, d, d, d, d, d, d, d]
        L.orc_diff_backward.restype = ctypes.c_double
        L.orc_diff_source_validity.argtypes = [dp, d, d, d, d, d, u8]
        L.orc_diff_forward_frozen.argtypes = [dp, d, d, d, d, d, d, u8]
        L.orc_diff_forward_frozen.restype = ctypes.c_double
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray, ctype):
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the oracle must be C-contiguous"
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def compose_homography(K, Rl, Tl, Rr, Tr) -> np.ndarray:
    """a1: 12 doubles, H1 (row-major) then H2 (stereo_mapper.cpp:79-80)."""
    out = np.zeros(12, np.float64)
    lib().orc_compose_homography(*[_ptr(_f64(x).reshape(-1), ctypes.c_double)
                                   for x in (K, Rl, Tl, Rr, Tr)], _ptr(out, ctypes.c_double))
    return out


def relative_pose(R, t, Rprev, tprev) -> np.ndarray:
    out = np.zeros(12, np.float64)
    lib().orc_relative_pose(*[_ptr(_f64(x).reshape(-1), ctypes.c_double)
                              for x in (R, t, Rprev, tprev)], _ptr(out, ctypes.c_double))
    return out


def _dt(prec):
    return (np.float64, ctypes.c_double) if prec == "f64" else (np.float32, ctypes.c_float)


def calc_cost(p: Params, ref: np.ndarray, srcs: np.ndarray, homs: np.ndarray, prec="f64"):
    """a3: returns (cost, cnt) volumes of shape (H, W, D)."""
    dt, ct = _dt(prec)
    ref = np.ascontiguousarray(ref, np.uint8)
    srcs = np.ascontiguousarray(srcs, np.uint8).reshape(-1, p.H, p.W)
    homs = _f64(homs).reshape(-1, 12)
    assert homs.shape[0] == srcs.shape[0]
    cost = np.empty((p.H, p.W, p.D), dt)
    cnt = np.empty((p.H, p.W, p.D), dt)
    fn = lib().orc_calc_cost_f64 if prec == "f64" else lib().orc_calc_cost_f32
    fn(ctypes.byref(p.c()), _ptr(ref, ctypes.c_uint8), _ptr(srcs, ctypes.c_uint8),
       srcs.shape[0], _ptr(homs, ctypes.c_double), _ptr(cost, ct), _ptr(cnt, ct))
    return cost, cnt


def sgm(p: Params, ref: np.ndarray, cost: np.ndarray, prec="f64") -> np.ndarray:
    """a4: aggregated volume (H, W, D), sum over p.num_paths directions."""
    dt, ct = _dt(prec)
    ref = np.ascontiguousarray(ref, np.uint8)
    cost = np.ascontiguousarray(cost, dt)
    out = np.empty_like(cost)
    fn = lib().orc_sgm_f64 if prec == "f64" else lib().orc_sgm_f32
    fn(ctypes.byref(p.c()), _ptr(ref, ctypes.c_uint8), _ptr(cost, ct), _ptr(out, ct))
    return out


def filter_cost(p: Params, vol: np.ndarray, prec="f64"):
    """a5: (depth (H, W), WTA index (H, W))."""
    dt, ct = _dt(prec)
    vol = np.ascontiguousarray(vol, dt)
    depth = np.empty((p.H, p.W), dt)
    idx = np.empty((p.H, p.W), np.int32)
    fn = lib().orc_filter_f64 if prec == "f64" else lib().orc_filter_f32
    fn(ctypes.byref(p.c()), _ptr(vol, ct), _ptr(depth, ct), _ptr(idx, ctypes.c_int32))
    return depth, idx


# pm_stats word order of the fusion counters (orc_fuse_gpu_counts_f32 / orc_fuse_cpu_counts)
FUSION_COUNTS = ("tf_empty", "tf_outlier", "tf_behind", "tf_outside", "tf_moved",
                 "pred_none", "pred_copied", "pred_filled",
                 "upd_empty", "upd_init", "upd_no_measurement", "upd_output", "upd_hidden")
WTA_CLASSES = ("wta_depth", "wta_no_overlap", "wta_border", "wta_flat", "wta_ambiguous")


def filter_classes(p: Params, vol: np.ndarray):
    """a5 in FP32 with each pixel's outcome: (depth, index, class (H, W) uint8 in WTA_CLASSES order)."""
    vol = np.ascontiguousarray(vol, np.float32)
    depth = np.empty((p.H, p.W), np.float32)
    idx = np.empty((p.H, p.W), np.int32)
    cls = np.empty((p.H, p.W), np.uint8)
    lib().orc_filter_classes_f32(ctypes.byref(p.c()), _ptr(vol, ctypes.c_float), _ptr(depth, ctypes.c_float),
                                 _ptr(idx, ctypes.c_int32), _ptr(cls, ctypes.c_uint8))
    return depth, idx, cls


def tree_order(D: int, compat: int = 1):
    rank = np.empty(D, np.int32)
    incl = np.empty(D, np.int32)
    lib().orc_tree_order(D, compat, _ptr(rank, ctypes.c_int32), _ptr(incl, ctypes.c_int32))
    return rank, incl


@dataclass
class FusionState:
    alpha: np.ndarray
    beta: np.ndarray
    mu: np.ndarray
    sigma: np.ndarray

    @staticmethod
    def zeros(W, H, dt=np.float32):
        return FusionState(*[np.zeros(W * H, dt) for _ in range(4)])

    def copy(self):
        return FusionState(self.alpha.copy(), self.beta.copy(), self.mu.copy(), self.sigma.copy())


def fuse_gpu(W, H, pose12, cam4, depth, pre: FusionState, cur: FusionState, prec="f32", counts=None):
    """a6-a10: one depth_fuse call.  depth is updated in place and returned with the
    filled propagation table; pre is modified in place like transformMap does.  counts: an
    optional dict that receives the step's FUSION_COUNTS (FP32 only)."""
    dt, ct = _dt(prec)
    pose = np.ascontiguousarray(pose12, np.float32)
    cam = np.ascontiguousarray(cam4, np.float32)
    table = np.zeros(W * H, np.int32)
    for a in (depth, pre.alpha, pre.beta, pre.mu, pre.sigma, cur.alpha, cur.beta, cur.mu, cur.sigma):
        assert a.dtype == dt and a.flags["C_CONTIGUOUS"]
    args = [W, H, _ptr(pose, ctypes.c_float), _ptr(cam, ctypes.c_float), _ptr(depth, ct),
            _ptr(pre.alpha, ct), _ptr(pre.beta, ct), _ptr(pre.mu, ct), _ptr(pre.sigma, ct),
            _ptr(cur.alpha, ct), _ptr(cur.beta, ct), _ptr(cur.mu, ct), _ptr(cur.sigma, ct),
            _ptr(table, ctypes.c_int32)]
    if counts is not None:
        assert prec == "f32"
        c = np.zeros(len(FUSION_COUNTS), np.uint32)
        lib().orc_fuse_gpu_counts_f32(*args, _ptr(c, ctypes.c_uint32))
        counts.update(zip(FUSION_COUNTS, (int(v) for v in c)))
    else:
        (lib().orc_fuse_gpu_f64 if prec == "f64" else lib().orc_fuse_gpu_f32)(*args)
    return depth, table


def fuse_cpu(W, H, pose12, cam4, pre_index, result, state: dict, counts=None):
    """a13: outputFusionCPU for a non-first frame; state holds 'alpha','beta','mu','sigma'
    arrays of shape (2, H*W) float32 and 'table' (2, H*W) uint32.  counts: an optional dict that
    receives the step's FUSION_COUNTS."""
    pose = _f64(pose12)
    cam = np.ascontiguousarray(cam4, np.float32)
    result = np.ascontiguousarray(result, np.float32).reshape(-1)
    args = [W, H, _ptr(pose, ctypes.c_double), _ptr(cam, ctypes.c_float), int(pre_index),
            _ptr(result, ctypes.c_float), _ptr(state["alpha"], ctypes.c_float),
            _ptr(state["beta"], ctypes.c_float), _ptr(state["mu"], ctypes.c_float),
            _ptr(state["sigma"], ctypes.c_float), _ptr(state["table"], ctypes.c_uint32)]
    if counts is not None:
        c = np.zeros(len(FUSION_COUNTS), np.uint32)
        lib().orc_fuse_cpu_counts(*args, _ptr(c, ctypes.c_uint32))
        counts.update(zip(FUSION_COUNTS, (int(v) for v in c)))
    else:
        lib().orc_fuse_cpu(*args)
    return result


def convert(W, H, data: np.ndarray, flag: int, pitch_bytes: int) -> np.ndarray:
    """a11: flag=1 linear (H*W) -> pitched bytes (H*pitch); flag=0 the reverse."""
    src = np.ascontiguousarray(data)
    if flag:
        out = np.zeros(H * pitch_bytes, np.uint8)
    else:
        out = np.zeros(W * H, np.float32)
    lib().orc_convert(W, H, src.ctypes.data, out.ctypes.data, int(flag), int(pitch_bytes))
    return out


@dataclass
class Mapper:
    """StereoMapper orchestration (stereo_mapper.cpp:27-244, 625-820) over the oracle stages.
    fusion='gpu' follows outputFusion (depth_fusion.cu kernels); 'cpu' follows outputFusionCPU."""
    p: Params
    K: np.ndarray
    prec: str = "f64"
    fusion: str = "gpu"
    ref: np.ndarray = None
    srcs: list = field(default_factory=list)
    homs: list = field(default_factory=list)
    first: bool = True
    pre_index: int = 0
    R_prev: np.ndarray = None
    t_prev: np.ndarray = None
    gstate: list = None
    cstate: dict = None

    def init_reference(self, img):
        self.ref = np.ascontiguousarray(img, np.uint8)
        self.srcs, self.homs = [], []

    def update(self, img, Rl, Tl, Rr, Tr):
        self.srcs.append(np.ascontiguousarray(img, np.uint8))
        self.homs.append(compose_homography(self.K, Rl, Tl, Rr, Tr))

    def stages(self):
        p = self.p
        cost, cnt = calc_cost(p, self.ref, np.stack(self.srcs), np.stack(self.homs), self.prec)
        vol = sgm(p, self.ref, cost, self.prec)
        st = dict(cost=cost, cnt=cnt, sgm=vol)
        if self.prec == "f32":   # with the pm_stats counters of the step
            depth, idx, cls = filter_classes(p, vol)
            st["stats"] = {n: int(np.count_nonzero(cls == k)) for k, n in enumerate(WTA_CLASSES)}
            st["stats"].update((n, 0) for n in FUSION_COUNTS)
        else:
            depth, idx = filter_cost(p, vol, self.prec)
        st.update(depth=depth, idx=idx)
        return st

    def output(self):
        return self.stages()["depth"]

    def output_fusion(self, R, t, fx, fy, cx, cy):
        st = self.stages()
        W, H = self.p.W, self.p.H
        dt = np.float64 if (self.prec == "f64" and self.fusion == "gpu") else np.float32
        if self.first:
            self.first = False
            self.R_prev, self.t_prev = np.array(R, np.float64), np.array(t, np.float64)
            self.pre_index = 0
            if self.fusion == "gpu":
                self.gstate = [FusionState.zeros(W, H, dt), FusionState.zeros(W, H, dt)]
            else:
                self.cstate = {k: np.zeros((2, W * H), np.float32) for k in ("alpha", "beta", "mu", "sigma")}
                self.cstate["table"] = np.zeros((2, W * H), np.uint32)
            st["fused"] = np.zeros((H, W), dt)
            st["variance"] = np.zeros((H, W), dt)
            return st
        rel = relative_pose(R, t, self.R_prev, self.t_prev)
        cam = np.array([fx, fy, cx, cy], np.float32)
        if self.fusion == "gpu":
            pre = self.gstate[self.pre_index]
            cur = self.gstate[self.pre_index ^ 1]
            depth = np.ascontiguousarray(st["depth"], dt).reshape(-1).copy()
            fuse_gpu(W, H, rel.astype(np.float32), cam, depth, pre, cur, "f64" if dt == np.float64 else "f32",
                     counts=st.get("stats"))
            st["fused"] = depth.reshape(H, W)
            st["variance"] = cur.sigma.reshape(H, W).copy()
        else:
            res = np.ascontiguousarray(st["depth"], np.float32).reshape(-1).copy()
            fuse_cpu(W, H, rel, cam, self.pre_index, res, self.cstate, counts=st.get("stats"))
            st["fused"] = res.reshape(H, W)
            st["variance"] = self.cstate["sigma"][self.pre_index ^ 1].reshape(H, W).copy()
        self.R_prev, self.t_prev = np.array(R, np.float64), np.array(t, np.float64)
        self.pre_index ^= 1
        return st


# ---- differentiable form (pm_oracle_diff.cpp) ---------------------------------------------
class OrcDiffParams(ctypes.Structure):
    _fields_ = [("W", ctypes.c_int), ("H", ctypes.c_int), ("D", ctypes.c_int), ("S", ctypes.c_int),
                ("num_paths", ctypes.c_int), ("rho0", ctypes.c_double), ("drho", ctypes.c_double),
                ("temperature", ctypes.c_double), ("p1", ctypes.c_double), ("p2", ctypes.c_double),
                ("tau_so", ctypes.c_double), ("q1", ctypes.c_double), ("q2", ctypes.c_double)]


@dataclass
class DiffParams:
    """The differentiable form: corrected 3x3 cost, 8 SGM paths, soft-argmin at temperature T,
    L1 loss against the ground-truth inverse depth."""
    W: int
    H: int
    D: int
    S: int
    rho0: float
    drho: float
    temperature: float = 0.05
    p1: float = 0.003
    p2: float = 0.01
    tau_so: float = 3.5 / 255
    q1: float = 2.0
    q2: float = 3.0
    num_paths: int = 8

    def c(self):
        return OrcDiffParams(self.W, self.H, self.D, self.S, self.num_paths, self.rho0, self.drho,
                             self.temperature, self.p1, self.p2, self.tau_so, self.q1, self.q2)


def _diff_args(p: DiffParams, ref, srcs, K, R, t, rho_gt):
    arrs = [_f64(ref).reshape(-1), _f64(srcs).reshape(-1), _f64(K).reshape(-1), _f64(R).reshape(-1),
            _f64(t).reshape(-1), _f64(rho_gt).reshape(-1)]
    assert arrs[1].size == p.S * p.W * p.H and arrs[3].size == 9 * p.S and arrs[4].size == 3 * p.S
    return arrs


def diff_forward(p: DiffParams, ref, srcs, K, R, t, rho_gt):
    """FP64 loss, rho_hat (H, W) and pixel validity of the differentiable form."""
    a = _diff_args(p, ref, srcs, K, R, t, rho_gt)
    rho_hat = np.zeros(p.W * p.H)
    valid = np.zeros(p.W * p.H, np.uint8)
    cp = p.c()
    loss = lib().orc_diff_forward(ctypes.byref(cp), *[_ptr(x, ctypes.c_double) for x in a],
                                  _ptr(rho_hat, ctypes.c_double), _ptr(valid, ctypes.c_uint8))
    return loss, rho_hat.reshape(p.H, p.W), valid.reshape(p.H, p.W)


def diff_source_validity(p: DiffParams, ref, srcs, K, R, t):
    """(H, W, D, S) uint8: 1 where source s measures plane d of the pixel at this pose."""
    a = _diff_args(p, ref, srcs, K, R, t, np.zeros(p.W * p.H))[:5]
    ok = np.zeros(p.W * p.H * p.D * p.S, np.uint8)
    cp = p.c()
    lib().orc_diff_source_validity(ctypes.byref(cp), *[_ptr(x, ctypes.c_double) for x in a], _ptr(ok, ctypes.c_uint8))
    return ok.reshape(p.H, p.W, p.D, p.S)


def diff_forward_frozen(p: DiffParams, ref, srcs, K, R, t, rho_gt, frozen):
    """FP64 loss with the source validity flags held at `frozen` (diff_source_validity of the base
    pose): the loss as a function of the pose without border jumps."""
    a = _diff_args(p, ref, srcs, K, R, t, rho_gt)
    fz = np.ascontiguousarray(frozen, np.uint8).reshape(-1)
    assert fz.size == p.W * p.H * p.D * p.S
    cp = p.c()
    return lib().orc_diff_forward_frozen(ctypes.byref(cp), *[_ptr(x, ctypes.c_double) for x in a],
                                         _ptr(fz, ctypes.c_uint8))


def diff_backward(p: DiffParams, ref, srcs, K, R, t, rho_gt):
    """FP64 loss and its gradients: w.r.t. the source images (S, H, W) and w.r.t. the left se(3)
    perturbation (omega, upsilon) of each source pose (S, 6)."""
    a = _diff_args(p, ref, srcs, K, R, t, rho_gt)
    g_srcs = np.zeros(p.S * p.W * p.H)
    g_pose = np.zeros(6 * p.S)
    cp = p.c()
    loss = lib().orc_diff_backward(ctypes.byref(cp), *[_ptr(x, ctypes.c_double) for x in a],
                                   _ptr(g_srcs, ctypes.c_double), _ptr(g_pose, ctypes.c_double))
    return loss, g_srcs.reshape(p.S, p.H, p.W), g_pose.reshape(p.S, 6)


def so3_exp(w):
    """Rodrigues' formula, FP64."""
    w = np.asarray(w, np.float64)
    th = np.linalg.norm(w)
    Wx = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    if th < 1e-12:
        return np.eye(3) + Wx
    return np.eye(3) + np.sin(th) / th * Wx + (1 - np.cos(th)) / th ** 2 * (Wx @ Wx)


def perturb_pose(R, t, xi):
    """Left se(3) perturbation of a source-from-reference pose: P -> exp([omega]) P + upsilon."""
    E = so3_exp(xi[:3])
    return E @ R, E @ t + np.asarray(xi[3:], np.float64)
