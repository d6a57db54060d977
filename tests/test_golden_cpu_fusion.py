"""The CPU fusion variant of the oracle against the reference's OWN code.

tests/golden/ref_cpu_fusion_80x60x32.npz holds the outputs of the reference's
StereoMapper::outputFusionCPU (stereo_mapper.cpp:625-820: transformMapCPU, holeFillingCPU,
depthPreditCPU, depthUpdateCPU, depthFuseCPU and the masks, plus the CASE 0 / CASE 1 argmin),
compiled unmodified on the host (tests/golden/make_ref_cpu_golden.py).  Here, without a GPU:

 * oracle/imgproc.case_argmin reproduces the reference's CASE 0 and CASE 1 outputs bit for bit;
 * oracle.fuse_cpu, driven keyframe by keyframe as outputFusionCPU drives depthFuseCPU
   (first keyframe: zero state and a zero result; then the relative pose, the masks, the fusion
   and the ping-pong swap), reproduces every keyframe's fused result, every propagation table
   and the final state of both ping-pong halves.

The GPU kernels of the variant are checked against the same fixture in tests/test_gpu_fusion_cpu.py.
"""
import hashlib
import os
import sys

import numpy as np
import pytest

import oracle
from oracle import imgproc as oip

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_ref_cpu_golden as gold  # noqa: E402

FIXTURE = os.path.join(HERE, "golden", f"ref_cpu_fusion_{gold.W}x{gold.H}x{gold.D}.npz")


@pytest.fixture(scope="module")
def fixture():
    return dict(np.load(FIXTURE))


@pytest.fixture(scope="module")
def volumes(fixture):
    inp = gold.inputs()
    for k in ("cost0", "sgm0"):
        assert hashlib.sha256(inp[k].tobytes()).hexdigest() == fixture[f"in_{k}_sha256"].item().decode(), \
            f"the regenerated {k} volume differs from the one the fixture was made from"
    np.testing.assert_array_equal(inp["wta"], fixture["in_wta"])
    return inp


@pytest.mark.parametrize("case,vol", [(0, "cost0"), (1, "sgm0")])
def test_case_argmin_matches_reference(fixture, volumes, case, vol):
    v = volumes[vol].reshape(gold.H, gold.W, gold.D)
    # the reference's CASE depth is 1 / (index * DEP_SAMPLE): plane 0 at inverse depth 0
    dep, _ = oip.case_argmin(v, 0.0, float(fixture["in_dep_sample"]))
    want = fixture[f"ref_case{case}"]
    assert (dep.view(np.uint32) == want.view(np.uint32)).all()
    assert (want == 10000).any() or case == 1


def fuse_sequence(fixture):
    """oracle.fuse_cpu driven as outputFusionCPU drives depthFuseCPU; returns per-keyframe results
    and tables, and the final state."""
    W, H = gold.W, gold.H
    N = W * H
    K = fixture["in_K"]
    cam = np.array([K[0, 0], K[1, 1], K[0, 2], K[1, 2]], np.float32)
    state = {k: np.zeros((2, N), np.float32) for k in ("alpha", "beta", "mu", "sigma")}
    state["table"] = np.zeros((2, N), np.uint32)
    pre = 0
    results, tables = [], []
    R_prev = t_prev = None
    for k in range(fixture["in_wta"].shape[0]):
        R, t = fixture["in_R"][k], fixture["in_t"][k]
        if k == 0:
            results.append(np.zeros((H, W), np.float32))
            tables.append(np.zeros(N, np.uint32))
        else:
            rel = oracle.relative_pose(R, t, R_prev, t_prev)
            res = np.ascontiguousarray(fixture["in_wta"][k], np.float32).reshape(-1).copy()
            oracle.fuse_cpu(W, H, rel, cam, pre, res, state)
            results.append(res.reshape(H, W))
            tables.append(state["table"][pre ^ 1].copy())
            pre ^= 1
        R_prev, t_prev = R, t
    return results, tables, state, pre


def test_fusion_sequence_matches_reference(fixture):
    results, tables, state, pre = fuse_sequence(fixture)
    assert pre == int(fixture["ref_final_pre_index"])
    fused_px = 0
    for k, (got, want) in enumerate(zip(results, fixture["ref_fused"])):
        assert (tables[k] == fixture["ref_tables"][k]).all(), f"keyframe {k}: propagation table"
        assert (got.view(np.uint32) == want.view(np.uint32)).all(), \
            f"keyframe {k}: {int((got != want).sum())} fused values differ"
        fused_px += int((want != 0).sum())
    assert fused_px > 1000
    for i, name in enumerate(("alpha", "beta", "mu", "sigma")):
        assert (state[name].view(np.uint32) == fixture["ref_state"][i].view(np.uint32)).all(), name
