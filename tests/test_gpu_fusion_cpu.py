"""The CPU fusion variant (outputFusionCPU, stereo_mapper.cpp:625-820) run on the GPU against the
oracle's sequential FP32 restatement, over a keyframe sequence.

The GPU resolves the order-dependent z-buffer by replaying each cell's hitters in raster order,
so the propagation follows the sequential result exactly; the update uses CUDA's expf where the
oracle uses the host's expf, so depths, variances and states are compared within 1e-4
relative.
"""
import numpy as np
import pytest

import oracle
from probabilistic_mapping_b200 import _lib, scene
from probabilistic_mapping_b200.mapper import StereoMapper

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1])
def test_cpu_variant_sequence_matches_oracle(mode):
    W, H, D, S, F = 128, 96, 64, 3, 5
    seq = scene.make_sequence(W, H, 100.0, S, F, seed=61)
    rho0, drho = scene.plane_range(D)
    prm = dict(rho0=rho0, intensity_scale=1 / 255, num_paths=8, p1=0.003, p2=0.01, tau_so=3.5 / 255,
               uniqueness_ratio=0.95, cost_mode=mode)
    m = StereoMapper(W, H, D, fusion_variant=_lib.PM_FUSION_CPU_PATH, **prm)
    K = seq[0].K
    m.initIntrinsic(K, 0.0, drho)
    o = oracle.Mapper(oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=1 / 255, cost_mode=mode,
                                    num_paths=8, p1=0.003, p2=0.01, tau_so=3.5 / 255, uniqueness=0.95), K,
                      prec="f32", fusion="cpu")
    nonzero = 0
    for k, fs in enumerate(seq):
        m.initReference(fs.ref)
        o.init_reference(fs.ref)
        for s in range(S):
            m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
            o.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        got, var = m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
        st = o.output_fusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
        assert (m.wta_depth().view(np.uint32) == st["depth"].view(np.uint32)).all()
        if k == 0:
            assert (got == 0).all() and (var == 0).all()
            continue
        np.testing.assert_allclose(got, st["fused"], rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(var, st["variance"], rtol=1e-4, atol=1e-5)
        want = [o.cstate[n][o.pre_index] for n in ("alpha", "beta", "mu", "sigma")]
        for g, w in zip(m.get_state(), want):
            np.testing.assert_allclose(g, w, rtol=1e-4, atol=1e-5)
        nonzero += int((got != 0).sum())
    assert nonzero > 0
    m.close()


def test_fusion_step_times_640x480():
    """Measurement: the fusion step of both variants on the GPU (stage timer) at 640x480, next to
    the sequential restatement of outputFusionCPU on the host (the reference runs it as
    single-threaded CPU loops).  With PM_REPORT_DIR set the numbers go to
    $PM_REPORT_DIR/fusion_640x480.json."""
    import json
    import os
    import time
    W, H, D, S = 640, 480, 64, 3
    seq = scene.make_sequence(W, H, 520.0, S, 3, seed=71)
    rho0, drho = scene.plane_range(D)
    K = seq[0].K
    cam = (K[0, 0], K[1, 1], K[0, 2], K[1, 2])
    report = {}
    for name, variant in (("gpu_variant", _lib.PM_FUSION_GPU), ("cpu_variant", _lib.PM_FUSION_CPU_PATH)):
        m = StereoMapper(W, H, D, fusion_variant=variant, rho0=rho0, intensity_scale=1 / 255, p1=0.003, p2=0.01,
                         tau_so=3.5 / 255)
        m.initIntrinsic(K, 0.0, drho)
        m.enable_stage_timing(True)
        times = []
        for k, fs in enumerate(seq):
            m.initReference(fs.ref)
            for s in range(S):
                m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
            m.outputFusion(fs.R_ref, fs.T_ref, *cam)
            if k > 0:
                times.append(float(m.stage_times()[2]))
        report[name + "_ms"] = min(times)
        if variant == _lib.PM_FUSION_CPU_PATH:
            # the host restatement on the same inputs: the state before the last step and its WTA depth
            state = {n: np.zeros((2, W * H), np.float32) for n in ("alpha", "beta", "mu", "sigma")}
            state["table"] = np.zeros((2, W * H), np.uint32)
            for n, v in zip(("alpha", "beta", "mu", "sigma"), m.get_state()):
                state[n][0] = v
            depth = m.wta_depth().reshape(-1).copy()
            rel = oracle.relative_pose(seq[2].R_ref, seq[2].T_ref, seq[1].R_ref, seq[1].T_ref)
            t0 = time.perf_counter()
            oracle.fuse_cpu(W, H, rel, np.array(cam, np.float32), 0, depth, state)
            report["host_sequential_ms"] = 1000 * (time.perf_counter() - t0)
        m.close()
    print(json.dumps(report))
    out = os.environ.get("PM_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "fusion_640x480.json"), "w") as f:
            json.dump(report, f, indent=1)
    assert all(v > 0 for v in report.values())


def test_cpu_variant_kernels_match_the_reference_itself():
    """pm_stage_depth_fuse_cpu_path against the reference's own outputFusionCPU (compiled
    unmodified on the host; tests/golden/ref_cpu_fusion_80x60x32.npz) over a 6-keyframe sequence:
    every propagation table identical, every fused result and the final state within 1e-4
    relative (CUDA's expf against the host's), and identical wherever the update's
    transcendental does not enter (zero / non-fused pixels)."""
    import ctypes
    import os
    import torch
    from probabilistic_mapping_b200 import _lib as L
    lib = L.load()
    here = os.path.dirname(os.path.abspath(__file__))
    z = dict(np.load(os.path.join(here, "golden", "ref_cpu_fusion_80x60x32.npz")))
    F, H, W = z["in_wta"].shape
    N = W * H
    K = z["in_K"]
    cam = np.array([K[0, 0], K[1, 1], K[0, 2], K[1, 2]], np.float32)
    state = [[torch.zeros(N, dtype=torch.float32, device="cuda") for _ in range(4)] for _ in range(2)]
    table = torch.zeros(N, dtype=torch.int32, device="cuda")
    scratch = torch.empty(lib.pm_stage_depth_fuse_cpu_path_scratch(W, H), dtype=torch.uint8, device="cuda")
    pre = 0
    for k in range(F):
        if k == 0:
            continue   # the first keyframe only zeroes the state (done above)
        rel = oracle.relative_pose(z["in_R"][k], z["in_t"][k], z["in_R"][k - 1], z["in_t"][k - 1])
        res = torch.from_numpy(np.ascontiguousarray(z["in_wta"][k].reshape(-1))).cuda()
        prep = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in state[pre]])
        curp = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in state[pre ^ 1]])
        st = lib.pm_stage_depth_fuse_cpu_path(W, H, rel.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                              cam.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                              ctypes.c_void_p(res.data_ptr()), prep, curp,
                                              ctypes.c_void_p(table.data_ptr()), ctypes.c_void_p(scratch.data_ptr()),
                                              None)
        assert st == 0
        torch.cuda.synchronize()
        got = res.cpu().numpy().reshape(H, W)
        want = z["ref_fused"][k]
        assert (table.cpu().numpy().view(np.uint32) == z["ref_tables"][k]).all(), f"keyframe {k}: table"
        assert ((got == 0) == (want == 0)).all(), f"keyframe {k}: fused / rejected pixels differ"
        np.testing.assert_allclose(got, want, rtol=1e-4, atol=0, err_msg=f"keyframe {k}")
        pre ^= 1
    assert pre == int(z["ref_final_pre_index"])
    for h in range(2):
        for i, name in enumerate(("alpha", "beta", "mu", "sigma")):
            np.testing.assert_allclose(state[h][i].cpu().numpy(), z["ref_state"][i][h], rtol=1e-4, atol=1e-6,
                                       err_msg=f"{name}[{h}]")
