"""The differentiation form from Python: DepthLossEngine (the pm_diff_* C ABI) and DepthLoss, a
torch.autograd.Function whose backward runs the library's adjoint kernels.

The loss is the mean |rho_hat - rho_gt| over valid pixels, rho_hat the soft-argmin over the SGM
sum of the plane-sweep cost (see include/pm_stereo.h).  Gradients flow to the source images and
to a left se(3) perturbation xi = (omega, upsilon) of every source pose:
P_s -> exp([omega]) P_s + upsilon, P_s = R_s P_ref + t_s.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import load


def so3_exp(w):
    """Rodrigues' formula (FP64)."""
    w = np.asarray(w, np.float64)
    th = np.linalg.norm(w)
    Wx = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    if th < 1e-12:
        return np.eye(3) + Wx
    return np.eye(3) + np.sin(th) / th * Wx + (1 - np.cos(th)) / th ** 2 * (Wx @ Wx)


def perturb_pose(R, t, xi):
    """Left se(3) perturbation of a source-from-reference pose: P -> exp([omega]) P + upsilon."""
    E = so3_exp(np.asarray(xi[:3], np.float64))
    return E @ np.asarray(R, np.float64), E @ np.asarray(t, np.float64) + np.asarray(xi[3:], np.float64)


def _dp(a):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    return a, ctypes.cast(a.ctypes.data, ctypes.POINTER(ctypes.c_double))


class DepthLossEngine:
    def __init__(self, width, height, num_planes, num_sources, store_paths=False, device=0, **params):
        self.lib = load()
        c = _lib.PmDiffConfig()
        self.lib.pm_diff_config_default(ctypes.byref(c), width, height, num_planes, num_sources)
        c.store_paths = int(store_paths)
        c.device = device
        for k, v in params.items():
            if not hasattr(c, k):
                raise TypeError(f"unknown parameter {k}")
            setattr(c, k, v)
        self.cfg = c
        h = ctypes.c_void_p()
        _lib.check(self.lib.pm_diff_create(ctypes.byref(c), ctypes.byref(h)), None, "pm_diff_create")
        self.h = h
        self.W, self.H, self.D, self.S = width, height, num_planes, num_sources
        self._keep = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.pm_diff_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != 0:
            msg = self.lib.pm_diff_last_error(self.h)
            raise _lib.PmError(st, f"{what}: {msg.decode() if msg else ''}")

    def memory(self) -> int:
        b = ctypes.c_size_t()
        self._check(self.lib.pm_diff_memory(self.h, ctypes.byref(b)), "pm_diff_memory")
        return b.value

    def forward(self, ref, srcs, K, R, t, rho_gt):
        """ref (H, W), srcs (S, H, W), rho_gt (H, W): float32 CUDA tensors; K 3x3, R (S, 3, 3),
        t (S, 3) host arrays.  Returns (loss, rho_hat)."""
        import torch
        for x in (ref, srcs, rho_gt):
            assert x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()
        rho_hat = torch.empty_like(rho_gt)
        k, kp = _dp(K)
        r, rp = _dp(R)
        tt, tp = _dp(t)
        loss = ctypes.c_double()
        stream = torch.cuda.current_stream().cuda_stream
        self._check(self.lib.pm_diff_forward(self.h, ctypes.c_void_p(ref.data_ptr()), ctypes.c_void_p(srcs.data_ptr()),
                                             kp, rp, tp, ctypes.c_void_p(rho_gt.data_ptr()),
                                             ctypes.c_void_p(rho_hat.data_ptr()), ctypes.byref(loss),
                                             ctypes.c_void_p(stream)), "pm_diff_forward")
        self._keep = (ref, srcs, rho_gt)   # the backward reads them
        return loss.value, rho_hat

    def backward(self):
        """Gradients of the last forward's loss: (source images, CUDA tensor (S, H, W); poses,
        numpy (S, 6) as (omega, upsilon))."""
        import torch
        g = torch.empty((self.S, self.H, self.W), dtype=torch.float32, device="cuda")
        gp = np.zeros(6 * self.S)
        stream = torch.cuda.current_stream().cuda_stream
        self._check(self.lib.pm_diff_backward(self.h, ctypes.c_void_p(g.data_ptr()),
                                              gp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                              ctypes.c_void_p(stream)), "pm_diff_backward")
        return g, gp.reshape(self.S, 6)


def _autograd_function():
    import torch

    class DepthLoss(torch.autograd.Function):
        """loss = DepthLoss.apply(srcs, xi, engine, ref, K, R0, t0, rho_gt).  srcs: (S, H, W) CUDA
        float32; xi: (S, 6) left se(3) perturbations applied to the base poses (R0, t0).  The
        pose gradient is the derivative with respect to a further left perturbation at the
        perturbed pose, which is d loss / d xi exactly at xi = 0."""

        @staticmethod
        def forward(ctx, srcs, xi, engine, ref, K, R0, t0, rho_gt):
            x = xi.detach().cpu().double().numpy()
            R = np.stack([perturb_pose(R0[s], t0[s], x[s])[0] for s in range(len(R0))])
            t = np.stack([perturb_pose(R0[s], t0[s], x[s])[1] for s in range(len(R0))])
            loss, _ = engine.forward(ref, srcs.detach().contiguous(), K, R, t, rho_gt)
            ctx.engine = engine
            ctx.xi_dtype, ctx.xi_device = xi.dtype, xi.device
            return torch.tensor(loss, dtype=torch.float64, device=srcs.device)

        @staticmethod
        def backward(ctx, grad):
            g_src, g_pose = ctx.engine.backward()
            gs = g_src * grad.to(g_src.device, g_src.dtype)
            gp = torch.from_numpy(g_pose).to(ctx.xi_device, ctx.xi_dtype) * grad.to(ctx.xi_device, ctx.xi_dtype)
            return gs, gp, None, None, None, None, None, None

    return DepthLoss


_DEPTH_LOSS = None


def depth_loss(srcs, xi, engine, ref, K, R0, t0, rho_gt):
    """Functional form of DepthLoss.apply."""
    global _DEPTH_LOSS
    if _DEPTH_LOSS is None:
        _DEPTH_LOSS = _autograd_function()
    return _DEPTH_LOSS.apply(srcs, xi, engine, ref, K, R0, t0, rho_gt)
