"""Child process of tests/test_gpu_bounds.py: runs the motion-stereo path on odd shapes through
the library that PM_STEREO_LIB names (the product or the bounds-checked build) and saves every
output, plus the bounds record when the library keeps one, to the .npz given as argv[1].

Covered: the plain mapper (FP32 exact and texture, FP16 exact and texture, 4 and 8 paths, both
cost modes, incremental cost passes with more sources than max_sources), both fusion variants,
the CASE debug outputs, pixel counters, and the batched form (CUDA graph and persistent kernel)."""
import ctypes
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from probabilistic_mapping_b200 import _lib, scene  # noqa: E402
from probabilistic_mapping_b200.batch import StereoBatch  # noqa: E402
from probabilistic_mapping_b200.mapper import StereoMapper  # noqa: E402

S, F = 3, 3
COMMON = dict(intensity_scale=1 / 255, p1=0.003, p2=0.01, tau_so=3.5 / 255, uniqueness_ratio=0.95)
MAPPERS = [   # width, height, planes, precision, sampler, cost mode, paths, fusion variant, max sources
    (97, 61, 64, 0, 0, 0, 8, 0, 2),
    (130, 75, 128, 1, 2, 1, 4, 1, 8),
    (64, 33, 64, 1, 0, 0, 8, 0, 2),
    (101, 47, 96, 0, 2, 0, 8, 1, 8),
    (70, 90, 64, 1, 1, 0, 8, 0, 8),
    (45, 37, 192, 0, 0, 1, 8, 0, 8),    # six planes per lane, planes left out of the reduction tree
    (52, 29, 256, 1, 2, 0, 4, 1, 2),    # eight planes per lane, FP16, incremental passes
]


def main(out_path):
    out = {}
    for n, (W, H, D, prec, samp, mode, paths, fv, ms) in enumerate(MAPPERS):
        rho0, drho = scene.plane_range(D)
        seq = scene.make_sequence(W, H, 0.8 * W, S, F, seed=300 + n)
        m = StereoMapper(W, H, D, rho0=rho0, precision=prec, sampler=samp, cost_mode=mode, num_paths=paths,
                         fusion_variant=fv, max_sources=ms, **COMMON)
        K = seq[0].K
        m.initIntrinsic(K, 0.0, drho)
        m.enable_stats(True)
        for k, fs in enumerate(seq):
            m.initReference(fs.ref)
            for s in range(S):
                m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
            if k == 1:
                for case in (0, 1):
                    out[f"m{n}_case{case}"] = m.outputCase(case).copy()
                    for s in range(S):   # the same frames again: a mean over twice the sources
                        m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
            d, v = m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
            out[f"m{n}_k{k}_wta"] = m.wta_depth().copy()
            out[f"m{n}_k{k}_idx"] = m.wta_index().copy()
            out[f"m{n}_k{k}_fused"] = d.copy()
            out[f"m{n}_k{k}_var"] = v.copy()
            out[f"m{n}_k{k}_stats"] = np.array(list(m.stats().values()), np.uint32)
        m.close()
    for persistent in (False, True):
        cfgs = []
        for W, H, D in ((97, 61, 64), (130, 75, 128)):
            rho0, _ = scene.plane_range(D)
            cfgs.append(dict(width=W, height=H, num_planes=D, rho0=rho0, precision=1, sampler=2, cost_mode=0,
                             num_paths=8, **COMMON))
        seqs = [scene.make_sequence(c["width"], c["height"], 0.8 * c["width"], S, 2, seed=400 + i)
                for i, c in enumerate(cfgs)]
        b = StereoBatch(cfgs, S, lanes=0, host_io=True, persistent=persistent, stats=True)
        for i, c in enumerate(cfgs):
            _, drho = scene.plane_range(c["num_planes"])
            b.init_intrinsic(i, seqs[i][0].K, drho)
        for step in range(2):
            for i in range(len(cfgs)):
                fs = seqs[i][step]
                b.set_frame(i, 0, fs.ref)
                for s in range(S):
                    b.set_frame(i, 1 + s, fs.srcs[s])
                b.set_poses(i, fs.R_ref, fs.T_ref, list(fs.R_srcs), list(fs.T_srcs))
            b.run()
            b.synchronize()
            for i in range(len(cfgs)):
                d, v = b.output(i)
                out[f"b{int(persistent)}_{i}_{step}_fused"] = d.copy()
                out[f"b{int(persistent)}_{i}_{step}_var"] = v.copy()
                out[f"b{int(persistent)}_{i}_{step}_wta"] = b.wta_depth(i).copy()
                out[f"b{int(persistent)}_{i}_{step}_stats"] = np.array(list(b.stats(i).values()), np.uint32)
        b.close()
    lib = _lib.load()
    rec = (ctypes.c_uint64 * 4)()
    st = lib.pm_debug_bounds(rec, 1)
    out["bounds_status"] = np.array([st], np.int64)
    out["bounds"] = np.array(list(rec), np.uint64)
    np.savez_compressed(out_path, **out)


if __name__ == "__main__":
    main(sys.argv[1])
