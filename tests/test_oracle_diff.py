"""The FP64 transcription of the differentiable form against FP64 central finite differences.

The loss (corrected 3x3 cost, 8 SGM paths, soft-argmin at T = 0.05, L1 to the ground-truth
inverse depth) is piecewise smooth: the SGM minima, the absolute differences and the bilinear
cells switch at kinks, and a warped sample that crosses the image border drops a source from a
voxel's mean -- a jump.  Central differences with a step of 1e-5 on source intensities move no
sample and match the adjoint to ~1e-9; a pose step moves every sample, and at 1e-5 a few border
crossings already add jumps, so the pose is checked with a step of 1e-7 -- and at the step of
1e-5 with the validity of each (pixel, plane, source) held at the base pose
(orc_diff_forward_frozen), which removes the jumps and leaves only the kinks.
"""
import numpy as np
import pytest

import oracle
from probabilistic_mapping_b200 import scene

W, H, D, S = 48, 32, 16, 2


@pytest.fixture(scope="module")
def case(oracle_lib):
    fs = scene.make_frameset(W, H, 0.8 * W, S, seed=5)
    rho0, drho = scene.plane_range(D)
    p = oracle.DiffParams(W=W, H=H, D=D, S=S, rho0=rho0, drho=drho)
    ref = fs.ref / 255.0
    srcs = np.stack([fs.srcs[s] / 255.0 for s in range(S)])
    R = np.stack([fs.R_srcs[s].T @ fs.R_ref for s in range(S)])
    t = np.stack([fs.R_srcs[s].T @ (fs.T_ref - fs.T_srcs[s]) for s in range(S)])
    return p, ref, srcs, fs.K, R, t, 1.0 / fs.gt_depth


def test_forward_and_backward_agree_on_the_loss(case):
    p, ref, srcs, K, R, t, rgt = case
    l1, rho_hat, valid = oracle.diff_forward(p, ref, srcs, K, R, t, rgt)
    l2, _, _ = oracle.diff_backward(p, ref, srcs, K, R, t, rgt)
    assert l1 == l2 and l1 > 0
    assert valid.mean() > 0.5
    assert ((rho_hat > 0) == (valid > 0)).all()


def test_intensity_gradient_matches_central_differences(case):
    p, ref, srcs, K, R, t, rgt = case
    _, gi, _ = oracle.diff_backward(p, ref, srcs, K, R, t, rgt)
    eps = 1e-5
    for k in np.argsort(-np.abs(gi.reshape(-1)))[:6]:
        s, rem = divmod(int(k), W * H)
        y, x = divmod(rem, W)
        sp = srcs.copy()
        sp[s, y, x] += eps
        sm = srcs.copy()
        sm[s, y, x] -= eps
        fd = (oracle.diff_forward(p, ref, sp, K, R, t, rgt)[0] - oracle.diff_forward(p, ref, sm, K, R, t, rgt)[0]) / (2 * eps)
        assert fd == pytest.approx(gi[s, y, x], rel=1e-6)


def test_pose_gradient_matches_central_differences(case):
    p, ref, srcs, K, R, t, rgt = case
    _, _, gp = oracle.diff_backward(p, ref, srcs, K, R, t, rgt)
    eps = 1e-7
    fd = np.zeros_like(gp)
    for s in range(S):
        for i in range(6):
            out = []
            for sign in (1, -1):
                xi = np.zeros(6)
                xi[i] = sign * eps
                Rq, tq = R.copy(), t.copy()
                Rq[s], tq[s] = oracle.perturb_pose(R[s], t[s], xi)
                out.append(oracle.diff_forward(p, ref, srcs, K, Rq, tq, rgt)[0])
            fd[s, i] = (out[0] - out[1]) / (2 * eps)
    np.testing.assert_allclose(gp, fd, rtol=1e-4, atol=1e-6)


def test_pose_gradient_matches_frozen_validity_differences_at_1e5():
    """Step 1e-5 with the sources of each voxel held fixed: no border jumps, only the kinks of
    the SGM minima, the absolute differences and the bilinear cells, which the step crosses on
    a fraction of the samples (0.9 % L2 here; 40x without the freeze)."""
    W2, H2, D2 = 128, 96, 32
    fs = scene.make_frameset(W2, H2, 100.0, S, seed=5)
    rho0, drho = scene.plane_range(D2)
    p = oracle.DiffParams(W=W2, H=H2, D=D2, S=S, rho0=rho0, drho=drho)
    ref = fs.ref / 255.0
    srcs = np.stack([fs.srcs[s] / 255.0 for s in range(S)])
    R = np.stack([fs.R_srcs[s].T @ fs.R_ref for s in range(S)])
    t = np.stack([fs.R_srcs[s].T @ (fs.T_ref - fs.T_srcs[s]) for s in range(S)])
    rgt = 1.0 / fs.gt_depth
    _, _, gp = oracle.diff_backward(p, ref, srcs, fs.K, R, t, rgt)
    frozen = oracle.diff_source_validity(p, ref, srcs, fs.K, R, t)
    assert 0.5 < frozen.mean() < 1.0   # some sources do leave the image
    assert oracle.diff_forward_frozen(p, ref, srcs, fs.K, R, t, rgt, frozen) == \
        oracle.diff_forward(p, ref, srcs, fs.K, R, t, rgt)[0]
    eps = 1e-5
    fd = np.zeros_like(gp)
    for s in range(S):
        for i in range(6):
            out = []
            for sign in (1, -1):
                xi = np.zeros(6)
                xi[i] = sign * eps
                Rq, tq = R.copy(), t.copy()
                Rq[s], tq[s] = oracle.perturb_pose(R[s], t[s], xi)
                out.append(oracle.diff_forward_frozen(p, ref, srcs, fs.K, Rq, tq, rgt, frozen))
            fd[s, i] = (out[0] - out[1]) / (2 * eps)
    assert np.linalg.norm(fd - gp) / np.linalg.norm(gp) < 0.02
