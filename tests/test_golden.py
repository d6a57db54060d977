"""The oracle against the reference's own CUDA (tests/golden/ref_40x32x32.npz).

The fixture holds inputs and outputs of the reference's ad_calc_cost, sgm2, filter_cost,
depth_fuse and convert (motion_stereo/*.cu), built unmodified for sm_100a through a
texture-object shim and run on a B200 by tests/golden/make_ref_golden.py.  Case A uses the
reference parameters on 0..255 intensities (parameters.cpp:12-18), case B the scaled intensities
and penalties of the benchmark.  What is pinned here, and how tightly:

* sgm2 (sgm.cu): the FP32 oracle in the reference's path order is bit-exact.
* filter_cost (filter_cost.cu): FP32 oracle bit-exact (index, subpixel, depth).
* ad_calc_cost: validity and per-plane source counts exact; values within the texture unit's
  bilinear weight quantisation (9-bit fixed-point weights, not reproducible in FP arithmetic).
* depth_fuse: transformMap's in-place edits bit-exact; every z-buffer winner exact; hole filling
  is a race in the reference, the deterministic rule agrees on most filled cells; the update
  differs from CUDA's expf/rsqrtf by ulps on the CPU.
* convert: bit-exact.
"""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_40x32x32.npz")
W, H, D = 40, 32, 32


@pytest.fixture(scope="module")
def g():
    return dict(np.load(GOLDEN))


def params(g, case, **kw):
    sc, p1, p2, tau, q1, q2, vs = g[f"{case}_params"]
    return oracle.Params(W=W, H=H, D=D, drho=float(g["dep_sample"]), rho0=0.0,
                         intensity_scale=float(np.float32(sc)), num_paths=4, p1=p1, p2=p2, tau_so=tau,
                         q1=q1, q2=q2, var_scale=vs, tree_compat=1, cost_mode=0, **kw)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("case", ["A", "B"])
@pytest.mark.parametrize("quant", [0, 1])
def test_calc_cost_matches_reference(oracle_lib, g, case, quant):
    p = params(g, case, bilinear_quant=quant)
    cost, cnt = oracle.calc_cost(p, g["ref_u8"], g["srcs_u8"], g["homs"].astype(np.float64), "f64")
    rc, rn = g[f"{case}_cost"], g[f"{case}_cnt"]
    assert (cnt.astype(np.uint8) == rn).all()
    assert ((cost >= 0) == (rc >= 0)).all()
    both = (cost >= 0) & (rc >= 0)
    assert both.mean() > 0.5
    rel = np.abs(cost[both] - rc[both]) / np.maximum(rc[both], 1e-6)
    # texture-unit weights are 8-bit fractions: exact weights differ by up to 2^-9 per axis
    assert np.percentile(rel, 99) < (1.5e-3 if quant == 0 else 1e-3)
    assert np.median(rel) < (2.5e-4 if quant == 0 else 1.2e-4)
    # and never more than a tenth of an intensity level
    assert np.abs(cost[both] - rc[both]).max() < 0.1 * p.intensity_scale


@pytest.mark.parametrize("case", ["A", "B"])
def test_sgm_bit_exact_with_reference(oracle_lib, g, case):
    p = params(g, case, sum_order=0)
    got = oracle.sgm(p, g["ref_u8"], g[f"{case}_cost"].astype(np.float32), "f32")
    assert (bits(got) == bits(g[f"{case}_sgm"])).all()
    # the FP64 oracle agrees to rounding
    got64 = oracle.sgm(p, g["ref_u8"], g[f"{case}_cost"].astype(np.float64), "f64")
    np.testing.assert_allclose(got64, g[f"{case}_sgm"], rtol=1e-5, atol=1e-4 * float(g[f"{case}_params"][0]))


@pytest.mark.parametrize("case", ["A", "B"])
def test_filter_bit_exact_with_reference(oracle_lib, g, case):
    p = params(g, case)
    depth, _ = oracle.filter_cost(p, g[f"{case}_sgm"].astype(np.float32), "f32")
    want = g[f"{case}_depth"]
    assert (bits(depth) == bits(want)).all()
    # all branches of filter_cost.cu:37-52 occur in the fixture
    assert (want == 0).any() and ((want > 0) & (want < 1000)).any()


def fuse_oracle(g):
    pre = oracle.FusionState(*[g["fuse_pre_in"][k].copy() for k in range(4)])
    cur = oracle.FusionState(*[g["fuse_cur_in"][k].copy() for k in range(4)])
    depth, table = oracle.fuse_gpu(W, H, g["fuse_pose"], g["fuse_cam"], g["fuse_depth_in"].copy(), pre, cur, "f32")
    return pre, cur, depth, table


def test_depth_fuse_matches_reference(oracle_lib, g):
    pre, cur, depth, table = fuse_oracle(g)
    rt = g["fuse_table"]
    # transformMap (depth_fusion.cu:8-78) edits the previous state in place: bit-exact
    for k, a in enumerate((pre.alpha, pre.beta, pre.mu, pre.sigma)):
        assert (bits(a) == bits(g["fuse_pre_out"][k])).all()
    # every cell some pixel projects to holds the nearest one, as in the reference
    moved = pre.mu != g["fuse_pre_in"][2]
    assert moved.sum() > 500
    hit = np.zeros(W * H, bool)
    cam = g["fuse_cam"].astype(np.float32)
    pose = g["fuse_pose"].astype(np.float32)
    for i in np.nonzero(moved)[0]:
        y, x = divmod(i, W)
        z = np.float64(g["fuse_pre_in"][2][i])
        P = pose[:9].astype(np.float64).reshape(3, 3) @ np.array([(x - cam[2]) / cam[0] * z,
                                                                  (y - cam[3]) / cam[1] * z, z]) + pose[9:]
        hit[int(P[1] / P[2] * cam[1] + cam[3] + 0.5) * W + int(P[0] / P[2] * cam[0] + cam[2] + 0.5)] = True
    assert (table[hit] == rt[hit]).all()
    # which neighbour fills a hole is a race in the reference (hole_filling, :80-105)
    assert ((table == 0) == (rt == 0)).all()
    agree = table == rt
    assert agree.mean() > 0.97
    # depthUpdate on the agreeing cells: equal to within CUDA's expf/rsqrtf ulps
    for k, a in enumerate((cur.alpha, cur.beta, cur.mu, cur.sigma)):
        r = g["fuse_cur_out"][k]
        np.testing.assert_allclose(a[agree], r[agree], rtol=1e-4, atol=1e-5)
        assert (bits(a[agree]) == bits(r[agree])).mean() > 0.9
    np.testing.assert_allclose(depth[agree], g["fuse_depth_out"][agree], rtol=1e-4, atol=1e-5)


def test_convert_bit_exact_with_reference(oracle_lib, g):
    got = oracle.convert(W, H, g["conv_in"], 1, 4 * (W + 5)).view(np.float32).reshape(H, W + 5)
    assert (bits(got[:, :W]) == bits(g["conv_out"][:, :W])).all()
