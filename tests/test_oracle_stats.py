"""The oracle's pm_stats classes (winner-take-all outcome per pixel, fusion counters per step).

These are the reference's own outcome branches (filter_cost.cu:37-51; transformMap / depth_predict /
depthUpdate, depth_fusion.cu:26-219; transformMapCPU / depthPreditCPU / depthUpdateCPU,
stereo_mapper.cpp:274-556), so the checks here are consistency checks against the maps the
same oracle writes: every pixel lands in exactly one class of each group, and each class
agrees with the value written for the pixel.
"""
import numpy as np
import pytest

import oracle
from probabilistic_mapping_b200 import scene

W, H, D, S = 64, 48, 64, 2


@pytest.fixture(scope="module")
def seq():
    return scene.make_sequence(W, H, 52.0, S, 4, seed=91)


def params(D=D):
    rho0, drho = scene.plane_range(D)
    return oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=1 / 255, num_paths=8, p1=0.003,
                         p2=0.01, tau_so=3.5 / 255, uniqueness=0.95)


def test_filter_classes_agree_with_the_written_depth(seq):
    p = params()
    fs = seq[0]
    homs = np.stack([oracle.compose_homography(fs.K, fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
                     for s in range(S)])
    cost, _ = oracle.calc_cost(p, fs.ref, fs.srcs, homs, "f32")
    vol = oracle.sgm(p, fs.ref, cost, "f32")
    depth, idx, cls = oracle.filter_classes(p, vol)
    d2, i2 = oracle.filter_cost(p, vol, "f32")
    assert (depth.view(np.uint32) == d2.view(np.uint32)).all() and (idx == i2).all()
    assert cls.max() < len(oracle.WTA_CLASSES)
    assert ((cls == 1) == (depth == 1000.0)).all()              # DEP_INF only for non-overlap
    assert (depth[cls == 0] > 0).all()                           # a depth for class 0 only
    assert (depth[cls >= 2] == 0).all()
    border = (idx == 0) | (idx == D - 1)
    assert (border[cls == 2]).all() and not border[(cls == 3) | (cls == 4) | (cls == 0)].any()
    for k in (0, 1, 3, 4):   # the scene reaches every class but the border plane
        assert (cls == k).any(), oracle.WTA_CLASSES[k]
    # without the uniqueness test no pixel is ambiguous, and the rest keep their class
    p0 = params()
    p0.uniqueness = 0.0
    _, _, c0 = oracle.filter_classes(p0, vol)
    assert not (c0 == 4).any() and (c0[cls != 4] == cls[cls != 4]).all()


@pytest.mark.parametrize("fusion", ["gpu", "cpu"])
def test_fusion_counters_partition_the_pixels(seq, fusion):
    p = params()
    o = oracle.Mapper(p, seq[0].K, prec="f32", fusion=fusion)
    K = seq[0].K
    N = W * H
    for k, fs in enumerate(seq):
        o.init_reference(fs.ref)
        for s in range(S):
            o.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        st = o.output_fusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
        c = st["stats"]
        assert sum(c[n] for n in oracle.WTA_CLASSES) == N
        tf = sum(c[n] for n in oracle.FUSION_COUNTS[:5])
        pred = c["pred_none"] + c["pred_copied"]
        upd = sum(c[n] for n in oracle.FUSION_COUNTS[8:])
        if k == 0:   # the first keyframe only initialises the state
            assert tf == pred == upd == 0
            continue
        assert tf == pred == upd == N
        assert c["pred_filled"] <= c["pred_copied"]
        if k == 1:   # nothing is confident yet: every cell starts from an empty state
            assert c["tf_empty"] == N and c["pred_none"] == N
            assert c["upd_empty"] + c["upd_init"] == N
            d = st["depth"].astype(np.float64)
            if fusion == "cpu":   # outputFusionCPU zeroes depths above 10 first (stereo_mapper.cpp:743-760)
                d = np.where(d > 10, 0.0, d)
            assert c["upd_init"] == int(np.count_nonzero(d >= 1e-5))
        else:
            assert c["tf_moved"] > 0 and c["pred_copied"] > 0
            assert c["upd_output"] + c["upd_hidden"] > 0
