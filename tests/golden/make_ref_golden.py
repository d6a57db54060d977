"""Generates tests/golden/ref_40x32x32.npz from the reference's own CUDA -- TEST INFRASTRUCTURE.

Runs on a GPU host with oracle/_ref/libref_40x32x32.so (the reference's motion_stereo/*.cu,
built unmodified by oracle/build_ref.py through the texture-object shim oracle/ref_shim.h).
Seeded synthetic inputs from probabilistic_mapping_b200.scene; outputs of the reference's
ad_calc_cost, sgm2, filter_cost, depth_fuse and convert are stored next to their inputs.

    python tests/golden/make_ref_golden.py [--out PATH] [--speed]

--speed also times the reference pipeline (libref_640x480x64.so, 5 sources, 4-path SGM,
reference parameters) and prints a JSON line; it is a same-GPU comparator, not a fixture.
"""
from __future__ import annotations

import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.join(ROOT, "tests", "golden", "ref_40x32x32.npz")


def load(W, H, D):
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", f"libref_{W}x{H}x{D}.so"))
    f = ctypes.POINTER(ctypes.c_float)
    i32 = ctypes.POINTER(ctypes.c_int32)
    lib.ref_set_params.argtypes = [ctypes.c_float] * 6
    lib.ref_calc_cost.argtypes = [f, f, ctypes.c_int, f, ctypes.c_float, f, f]
    lib.ref_sgm.argtypes = [f, f, f]
    lib.ref_filter.argtypes = [f, ctypes.c_float, f]
    lib.ref_depth_fuse.argtypes = [f, f, f, f, f, i32]
    lib.ref_convert.argtypes = [f, f, ctypes.c_int]
    lib.ref_bench.argtypes = [f, f, ctypes.c_int, f, ctypes.c_float, ctypes.c_int, f]
    return lib


def P(a, ct=ctypes.c_float):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ct))


def homographies(fs):
    import oracle
    return np.stack([oracle.compose_homography(fs.K, fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
                     for s in range(fs.srcs.shape[0])]).astype(np.float32)


CASES = {
    # reference parameters (parameters.cpp:12-18) on 0..255 intensities
    "A": dict(scale=1.0, p1=8.0, p2=24.0, tau=4.0, q1=2.0, q2=3.0, vs=1.02),
    # the bench's scaled intensities and penalties
    "B": dict(scale=1.0 / 255.0, p1=0.003, p2=0.01, tau=3.5 / 255.0, q1=2.0, q2=3.0, vs=1.02),
}


def make_fixture(out_path=OUT):
    from probabilistic_mapping_b200 import scene
    W, H, D, S = 40, 32, 32, 3
    lib = load(W, H, D)
    fs = scene.make_frameset(W, H, 0.8 * W, S, seed=123)
    dep_sample = np.float32(2.0 / (D - 1))
    homs = np.ascontiguousarray(homographies(fs))
    out = dict(ref_u8=fs.ref, srcs_u8=fs.srcs, homs=homs, dep_sample=dep_sample)
    for name, c in CASES.items():
        sc = np.float32(c["scale"])
        ref = np.ascontiguousarray(fs.ref.astype(np.float32) * sc)
        srcs = np.ascontiguousarray(fs.srcs.astype(np.float32) * sc)
        lib.ref_set_params(c["p1"], c["p2"], c["tau"], c["q1"], c["q2"], c["vs"])
        cost = np.empty((H, W, D), np.float32)
        cnt = np.empty((H, W, D), np.float32)
        assert lib.ref_calc_cost(P(ref), P(srcs), S, P(homs), dep_sample, P(cost), P(cnt)) == 0
        sgm = np.empty_like(cost)
        assert lib.ref_sgm(P(cost), P(ref), P(sgm)) == 0
        depth = np.empty((H, W), np.float32)
        assert lib.ref_filter(P(sgm), dep_sample, P(depth)) == 0
        out.update({f"{name}_cost": cost, f"{name}_cnt": cnt.astype(np.uint8), f"{name}_sgm": sgm,
                    f"{name}_depth": depth, f"{name}_params": np.array([c[k] for k in
                                                                        ("scale", "p1", "p2", "tau", "q1", "q2", "vs")])})
    # depth_fuse on a realistic previous state and the next frame's ground-truth-like depth
    seq = scene.make_sequence(W, H, 0.8 * W, 1, 2, seed=321)
    import oracle
    rng = np.random.default_rng(7)
    N = W * H
    pre = np.stack([rng.uniform(0.0, 20.0, N), rng.uniform(0.5, 12.0, N),
                    seq[0].gt_depth.reshape(-1) * rng.uniform(0.97, 1.03, N), rng.uniform(0.01, 3.0, N)]).astype(np.float32)
    pre[0][rng.uniform(size=N) < 0.1] = 0.0
    cur = np.full((4, N), 7.0, np.float32)
    depth = (seq[1].gt_depth.reshape(-1) * rng.uniform(0.95, 1.05, N)).astype(np.float32)
    depth[rng.uniform(size=N) < 0.1] = 0.0
    pose = oracle.relative_pose(seq[1].R_ref, seq[1].T_ref, seq[0].R_ref, seq[0].T_ref).astype(np.float32)
    K = seq[0].K
    cam = np.array([K[0, 0], K[1, 1], K[0, 2], K[1, 2]], np.float32)
    out.update(fuse_pose=pose, fuse_cam=cam, fuse_depth_in=depth.copy(), fuse_pre_in=pre.copy(),
               fuse_cur_in=cur.copy())
    table = np.zeros(N, np.int32)
    assert lib.ref_depth_fuse(P(pose), P(cam), P(depth), P(pre), P(cur), P(table, ctypes.c_int32)) == 0
    out.update(fuse_depth_out=depth, fuse_pre_out=pre, fuse_cur_out=cur, fuse_table=table)
    # convert, linear -> pitched with a pitch of W + 5 floats
    lin = np.arange(N, dtype=np.float32)
    pitched = np.zeros((H, W + 5), np.float32)
    assert lib.ref_convert(P(lin), P(pitched), W + 5) == 0
    out.update(conv_in=lin, conv_out=pitched)
    np.savez_compressed(out_path, **out)
    print(f"wrote {out_path} ({os.path.getsize(out_path)} bytes)")


def speed():
    """Reference pipeline at its native 640x480x64 (ad_calc_cost x5, sgm2, filter_cost) on this GPU."""
    from probabilistic_mapping_b200 import scene
    W, H, D, S = 640, 480, 64, 5
    lib = load(W, H, D)
    lib.ref_set_params(8.0, 24.0, 4.0, 2.0, 3.0, 1.02)
    fs = scene.make_frameset(W, H, 520.0, S, seed=99)
    ref = np.ascontiguousarray(fs.ref.astype(np.float32))
    srcs = np.ascontiguousarray(fs.srcs.astype(np.float32))
    homs = np.ascontiguousarray(homographies(fs))
    ms = np.zeros(1, np.float32)
    assert lib.ref_bench(P(ref), P(srcs), S, P(homs), np.float32(2.0 / (D - 1)), 20, P(ms)) == 0
    print(json.dumps({"reference_cuda_ms_per_map": float(ms[0]), "config": "640x480x64, 5 sources, 4-path SGM, "
                      "reference parameters, cost + sgm + filter (no fusion)"}))


if __name__ == "__main__":
    make_fixture(sys.argv[sys.argv.index("--out") + 1] if "--out" in sys.argv else OUT)
    if "--speed" in sys.argv:
        speed()
