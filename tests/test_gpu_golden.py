"""The CUDA kernels against the reference's own CUDA outputs (tests/golden/ref_40x32x32.npz).

Same fixture as test_golden.py, checked through the C ABI on the device:
* pm_stage_filter on the reference's SGM volume: bit-exact depth;
* pm_stage_sgm on the reference's cost volume: equal to the reference up to the order in which
  the four path sums are added (the kernels add them pairwise), bit-exact against the oracle
  in that order;
* pm_stage_calc_cost on the reference's inputs: same validity, values within the texture unit's
  bilinear weight quantisation; with the texture sampler (FP32 texels, the reference's own
  sampling) closer still;
* pm_stage_depth_fuse on the reference's inputs: transformMap edits bit-exact, z-buffer winners
  exact, and bit-exact updated state wherever the racy hole filling picked the same neighbour.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from test_golden import GOLDEN, D, H, W, params
from test_gpu_stages import bits, config, fptr, vp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def g():
    return dict(np.load(GOLDEN))


def scaled(g, key, scale):
    return torch.from_numpy(np.ascontiguousarray(g[key].astype(np.float32) * np.float32(scale))).cuda()


@pytest.mark.parametrize("case", ["A", "B"])
def test_filter_on_reference_sgm(pm_lib, g, case):
    p = params(g, case)
    vol = torch.from_numpy(g[f"{case}_sgm"]).cuda()
    depth = torch.empty((H, W), dtype=torch.float32, device="cuda")
    idx = torch.empty((H, W), dtype=torch.int32, device="cuda")
    cfg = config(p)
    assert pm_lib.pm_stage_filter(ctypes.byref(cfg), vp(vol), vp(depth), 4 * W, vp(idx), None) == 0
    torch.cuda.synchronize()
    assert (bits(depth.cpu().numpy()) == bits(g[f"{case}_depth"])).all()


@pytest.mark.parametrize("case", ["A", "B"])
def test_sgm_on_reference_cost(pm_lib, g, case):
    p = params(g, case)
    scale = float(g[f"{case}_params"][0])
    cost = torch.from_numpy(g[f"{case}_cost"]).cuda()
    ref = scaled(g, "ref_u8", scale)
    out = torch.empty_like(cost)
    part = torch.empty((p.num_paths - 1,) + tuple(cost.shape), dtype=torch.float32, device="cuda")
    cfg = config(p)
    assert pm_lib.pm_stage_sgm(ctypes.byref(cfg), vp(cost), vp(ref), vp(out), vp(part), None) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    p.sum_order = 1
    want = oracle.sgm(p, g["ref_u8"], g[f"{case}_cost"].astype(np.float32), "f32")
    assert (bits(got) == bits(want)).all()
    np.testing.assert_allclose(got, g[f"{case}_sgm"], rtol=2e-6, atol=1e-6 * scale)
    # the winner-take-all decision is the reference's on (almost) every pixel
    depth = torch.empty((H, W), dtype=torch.float32, device="cuda")
    idx = torch.empty((H, W), dtype=torch.int32, device="cuda")
    assert pm_lib.pm_stage_filter(ctypes.byref(cfg), vp(out), vp(depth), 4 * W, vp(idx), None) == 0
    torch.cuda.synchronize()
    # the reference's index: the (bit-exact) FP32 oracle filter on the reference's SGM volume
    _, ref_idx = oracle.filter_cost(p, g[f"{case}_sgm"].astype(np.float32), "f32")
    same = idx.cpu().numpy() == ref_idx
    assert same.mean() > 0.995
    # where the index agrees the subpixel depth differs only by the rounding of the sums
    np.testing.assert_allclose(depth.cpu().numpy()[same], g[f"{case}_depth"][same], rtol=1e-5)


@pytest.mark.parametrize("case", ["A", "B"])
def test_calc_cost_on_reference_inputs(pm_lib, g, case):
    p = params(g, case)
    scale = float(g[f"{case}_params"][0])
    ref = scaled(g, "ref_u8", scale)
    srcs = scaled(g, "srcs_u8", scale)
    S = srcs.shape[0]
    # the initReference state (cost -1, count 0) passed in explicitly, so the counts come back
    cost = torch.full((H, W, D), -1.0, dtype=torch.float32, device="cuda")
    cnt = torch.zeros((H, W, D), dtype=torch.float32, device="cuda")
    inv = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    hf = np.ascontiguousarray(g["homs"], np.float32).reshape(-1)
    cfg = config(p)
    st = pm_lib.pm_stage_calc_cost(ctypes.byref(cfg), vp(ref), vp(srcs), S, fptr(hf), vp(cost), vp(cnt),
                                   vp(inv), None)
    assert st == 0
    torch.cuda.synchronize()
    got = cost.cpu().numpy()
    rc = g[f"{case}_cost"]
    assert (cnt.cpu().numpy() == g[f"{case}_cnt"]).all()
    assert ((got >= 0) == (rc >= 0)).all()
    both = (got >= 0) & (rc >= 0)
    assert np.abs(got[both] - rc[both]).max() < 0.1 * scale
    rel = np.abs(got[both] - rc[both]) / np.maximum(rc[both], 1e-6)
    assert np.percentile(rel, 99) < 1.5e-3


def _stage_cost(pm_lib, g, case, sampler):
    p = params(g, case)
    scale = float(g[f"{case}_params"][0])
    ref = scaled(g, "ref_u8", scale)
    srcs = scaled(g, "srcs_u8", scale)
    cost = torch.full((H, W, D), -1.0, dtype=torch.float32, device="cuda")
    cnt = torch.zeros((H, W, D), dtype=torch.float32, device="cuda")
    hf = np.ascontiguousarray(g["homs"], np.float32).reshape(-1)
    cfg = config(p)
    cfg.sampler = sampler
    assert pm_lib.pm_stage_calc_cost(ctypes.byref(cfg), vp(ref), vp(srcs), srcs.shape[0], fptr(hf), vp(cost),
                                     vp(cnt), None, None) == 0
    torch.cuda.synchronize()
    return cost.cpu().numpy(), cnt.cpu().numpy()


@pytest.mark.parametrize("case", ["A", "B"])
def test_calc_cost_texture_sampler_on_reference_inputs(pm_lib, g, case):
    """The FP32 form with the reference's own sampler (PM_SAMPLER_TEXTURE_F32: the texture unit
    filters FP32 texels of the images, calc_cost.cu:226-237) reproduces the reference's cost volume
    more closely than the exact bilinear weights: same counts and validity, more voxels with
    identical bits, smaller typical difference.  With PM_REPORT_DIR set the figures go to
    $PM_REPORT_DIR/golden_cost_samplers_<case>.json."""
    import json
    from probabilistic_mapping_b200 import _lib
    scale = float(g[f"{case}_params"][0])
    rc = g[f"{case}_cost"]
    measured = rc >= 0
    report = {}
    for name, smp in (("exact", _lib.PM_SAMPLER_EXACT), ("texture_f32", _lib.PM_SAMPLER_TEXTURE_F32)):
        got, cnt = _stage_cost(pm_lib, g, case, smp)
        assert (cnt == g[f"{case}_cnt"]).all(), name
        assert ((got >= 0) == measured).all(), name
        diff = np.abs(got[measured].astype(np.float64) - rc[measured])
        rel = diff / np.maximum(rc[measured], 1e-6)
        report[name] = {"identical_bits": float((bits(got[measured]) == bits(rc[measured])).mean()),
                        "max_abs_diff_levels": float(diff.max() / scale),
                        "rel_median": float(np.median(rel)), "rel_p99": float(np.percentile(rel, 99))}
    print(json.dumps({case: report}))
    rep = os.environ.get("PM_REPORT_DIR")
    if rep:
        os.makedirs(rep, exist_ok=True)
        with open(os.path.join(rep, f"golden_cost_samplers_{case}.json"), "w") as f:
            json.dump(report, f, indent=1)
    ex, tx = report["exact"], report["texture_f32"]
    assert tx["identical_bits"] > ex["identical_bits"]
    assert tx["rel_p99"] < ex["rel_p99"]
    assert tx["max_abs_diff_levels"] < 0.5


def test_depth_fuse_on_reference_inputs(pm_lib, g):
    N = W * H
    d_pre = [torch.from_numpy(g["fuse_pre_in"][k].copy()).cuda() for k in range(4)]
    d_cur = [torch.from_numpy(g["fuse_cur_in"][k].copy()).cuda() for k in range(4)]
    d_depth = torch.from_numpy(g["fuse_depth_in"].copy()).cuda()
    zt = torch.empty(N, dtype=torch.int64, device="cuda")
    table = torch.empty(N, dtype=torch.int32, device="cuda")
    pose = np.ascontiguousarray(g["fuse_pose"], np.float32)
    cam = np.ascontiguousarray(g["fuse_cam"], np.float32)
    prep = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in d_pre])
    curp = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in d_cur])
    assert pm_lib.pm_stage_depth_fuse(W, H, fptr(pose), fptr(cam), vp(d_depth), prep, curp, vp(zt), vp(table),
                                      None) == 0
    torch.cuda.synchronize()
    for k in range(4):
        assert (bits(d_pre[k].cpu().numpy()) == bits(g["fuse_pre_out"][k])).all()
    t = table.cpu().numpy()
    rt = g["fuse_table"]
    # z-buffer winners (cells with a direct hit) are exact; a hole takes a racy neighbour
    direct = zt.cpu().numpy() != -1
    assert direct.sum() > 500
    assert (t[direct] == rt[direct]).all()
    assert ((t == 0) == (rt == 0)).all()
    agree = t == rt
    assert agree.mean() > 0.97
    for k in range(4):
        got = d_cur[k].cpu().numpy()
        want = g["fuse_cur_out"][k]
        assert (bits(got[agree]) == bits(want[agree])).mean() > 0.99, k
        np.testing.assert_allclose(got[agree], want[agree], rtol=1e-5, atol=1e-6)
    dd = d_depth.cpu().numpy()
    assert (bits(dd[agree]) == bits(g["fuse_depth_out"][agree])).mean() > 0.99
