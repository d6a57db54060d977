"""Differentiation form on the GPU (pm_diff_*) against the FP64 transcription and FP64 finite
differences.

Configuration: 320x240, 64 planes in [0.1, 2.0], 2 sources, f = 260, soft-argmin temperature
0.05, L1 loss against the ground-truth inverse depth of the seeded synthetic scene.
* loss: GPU (FP32) against the FP64 transcription, 1e-3 relative;
* gradients: GPU against the FP64 transcription's adjoint -- pose (12 values) within 2 % of the
  vector norm, source intensities within 5 % (relative L2) with correlation >= 0.99 (FP32
  sums and near-ties in the SGM minima move individual routes);
* FP64 central differences: intensities with a step of 1e-5; poses with a step of 1e-7, and with
  the step of 1e-5 on the loss whose per-voxel source validity is held at the base pose (a pose
  step moves every warped sample, and at 1e-5 samples crossing the image border switch sources
  in and out of a voxel's mean -- jumps of the loss; the plain 1e-5 pose differences are
  reported, not asserted);
* memory with and without per-path recomputation of the SGM states (same loss, same gradients
  up to the order of atomic sums), and the torch.autograd harness against the direct calls.
With PM_REPORT_DIR set the numbers go to $PM_REPORT_DIR/diff_320x240x64.json.
"""
import json
import os

import numpy as np
import pytest

import oracle
from probabilistic_mapping_b200 import scene
from probabilistic_mapping_b200.diff import DepthLossEngine, depth_loss, perturb_pose

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

W, H, D, S, F, T = 320, 240, 64, 2, 260.0, 0.05


@pytest.fixture(scope="module")
def case():
    fs = scene.make_frameset(W, H, F, S, seed=31)
    rho0, drho = scene.plane_range(D)
    ref = fs.ref / 255.0
    srcs = np.stack([fs.srcs[s] / 255.0 for s in range(S)])
    R = np.stack([fs.R_srcs[s].T @ fs.R_ref for s in range(S)])
    t = np.stack([fs.R_srcs[s].T @ (fs.T_ref - fs.T_srcs[s]) for s in range(S)])
    rgt = 1.0 / fs.gt_depth
    p = oracle.DiffParams(W=W, H=H, D=D, S=S, rho0=rho0, drho=drho, temperature=T)
    # the FP64 transcription sees the same FP32 values as the GPU
    ref32, srcs32, rgt32 = (np.float32(ref), srcs.astype(np.float32), rgt.astype(np.float32))
    return dict(p=p, K=fs.K, R=R, t=t, ref=ref32, srcs=srcs32, rgt=rgt32, rho0=rho0, drho=drho)


def gpu(case, store):
    e = DepthLossEngine(W, H, D, S, store_paths=store, rho0=case["rho0"], rho_step=case["drho"], temperature=T)
    ref = torch.from_numpy(case["ref"]).cuda()
    srcs = torch.from_numpy(case["srcs"]).cuda().contiguous()
    rgt = torch.from_numpy(case["rgt"]).cuda()
    loss, rho_hat = e.forward(ref, srcs, case["K"], case["R"], case["t"], rgt)
    gs, gp = e.backward()
    torch.cuda.synchronize()
    out = dict(loss=loss, rho_hat=rho_hat.cpu().numpy(), gs=gs.cpu().numpy(), gp=gp, mem=e.memory())
    e.close()
    return out


def oracle_loss(case, srcs=None, R=None, t=None):
    c = case
    return oracle.diff_forward(c["p"], c["ref"], c["srcs"] if srcs is None else srcs, c["K"],
                               c["R"] if R is None else R, c["t"] if t is None else t, c["rgt"])[0]


def test_diff_form(case):
    c = case
    g0 = gpu(case, store=False)
    g1 = gpu(case, store=True)
    # per-path recomputation changes memory, not results (the gradients' scatter and reductions
    # are atomic, so their summation order, and with it the last bits, varies from run to run)
    assert g0["loss"] == g1["loss"]
    np.testing.assert_allclose(g0["gs"], g1["gs"], rtol=1e-4, atol=1e-9)
    np.testing.assert_allclose(g0["gp"], g1["gp"], rtol=1e-4, atol=1e-9)
    assert g1["mem"] > g0["mem"]
    loss64, rh64, valid = oracle.diff_forward(c["p"], c["ref"], c["srcs"], c["K"], c["R"], c["t"], c["rgt"])
    assert g0["loss"] == pytest.approx(loss64, rel=1e-3)
    _, gs64, gp64 = oracle.diff_backward(c["p"], c["ref"], c["srcs"], c["K"], c["R"], c["t"], c["rgt"])
    pose_err = np.linalg.norm(g0["gp"] - gp64) / np.linalg.norm(gp64)
    img_err = np.linalg.norm(g0["gs"] - gs64) / np.linalg.norm(gs64)
    corr = np.corrcoef(g0["gs"].reshape(-1), gs64.reshape(-1))[0, 1]
    # FP64 central differences
    fd7 = np.zeros((S, 6))
    fd5 = np.zeros((S, 6))
    fd5f = np.zeros((S, 6))
    frozen = oracle.diff_source_validity(c["p"], c["ref"], c["srcs"], c["K"], c["R"], c["t"])
    for eps, fd, fz in ((1e-7, fd7, None), (1e-5, fd5, None), (1e-5, fd5f, frozen)):
        for s in range(S):
            for i in range(6):
                v = []
                for sign in (1, -1):
                    xi = np.zeros(6)
                    xi[i] = sign * eps
                    Rq, tq = c["R"].copy(), c["t"].copy()
                    Rq[s], tq[s] = perturb_pose(c["R"][s], c["t"][s], xi)
                    if fz is None:
                        v.append(oracle_loss(c, R=Rq, t=tq))
                    else:
                        v.append(oracle.diff_forward_frozen(c["p"], c["ref"], c["srcs"], c["K"], Rq, tq, c["rgt"], fz))
                fd[s, i] = (v[0] - v[1]) / (2 * eps)
    fd_err7 = np.linalg.norm(g0["gp"] - fd7) / np.linalg.norm(fd7)
    fd_err5 = np.linalg.norm(g0["gp"] - fd5) / np.linalg.norm(fd5)
    fd_err5f = np.linalg.norm(g0["gp"] - fd5f) / np.linalg.norm(fd5f)
    pix = []
    for k in np.argsort(-np.abs(gs64.reshape(-1)))[:5]:
        s, rem = divmod(int(k), W * H)
        y, x = divmod(rem, W)
        eps = 1e-5
        sp = c["srcs"].astype(np.float64)
        sp[s, y, x] += eps
        sm = c["srcs"].astype(np.float64)
        sm[s, y, x] -= eps
        fd = (oracle_loss(c, srcs=sp) - oracle_loss(c, srcs=sm)) / (2 * eps)
        pix.append((float(g0["gs"][s, y, x]), float(fd)))
    report = {"config": f"{W}x{H}, {D} planes, {S} sources, T={T}", "loss_gpu": g0["loss"], "loss_fp64": loss64,
              "pose_grad_rel_err_vs_fp64_adjoint": pose_err, "image_grad_rel_err_vs_fp64_adjoint": img_err,
              "image_grad_correlation": corr, "pose_grad_rel_err_vs_fd_step_1e-7": fd_err7,
              "pose_grad_rel_err_vs_fd_step_1e-5": fd_err5,
              "pose_grad_rel_err_vs_fd_step_1e-5_frozen_validity": fd_err5f, "image_grad_vs_fd_step_1e-5": pix,
              "device_bytes_recompute": g0["mem"], "device_bytes_store_paths": g1["mem"],
              "pose_grad_gpu": g0["gp"].tolist(), "pose_grad_fd_1e-7": fd7.tolist()}
    print(json.dumps(report))
    out = os.environ.get("PM_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "diff_320x240x64.json"), "w") as f:
            json.dump(report, f, indent=1)
    assert pose_err < 0.02
    assert img_err < 0.05 and corr > 0.99
    assert fd_err7 < 0.02
    assert fd_err5f < 0.02
    for a, b in pix:
        assert a == pytest.approx(b, rel=0.02, abs=1e-7)


def test_autograd_harness_matches_direct_calls(case):
    c = case
    e = DepthLossEngine(W, H, D, S, rho0=c["rho0"], rho_step=c["drho"], temperature=T)
    ref = torch.from_numpy(c["ref"]).cuda()
    rgt = torch.from_numpy(c["rgt"]).cuda()
    srcs = torch.from_numpy(c["srcs"]).cuda().requires_grad_(True)
    xi = torch.zeros((S, 6), dtype=torch.float64, requires_grad=True)
    loss = depth_loss(srcs, xi, e, ref, c["K"], c["R"], c["t"], rgt)
    (2.0 * loss).backward()
    _, gp = e.forward(ref, srcs.detach().contiguous(), c["K"], c["R"], c["t"], rgt)[0], None
    gs, gp = e.backward()
    torch.cuda.synchronize()
    torch.testing.assert_close(srcs.grad, 2.0 * gs, rtol=1e-4, atol=1e-9)
    np.testing.assert_allclose(xi.grad.numpy(), 2.0 * gp, rtol=1e-4, atol=1e-9)
    e.close()
