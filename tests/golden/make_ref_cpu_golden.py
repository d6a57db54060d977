"""Writes tests/golden/ref_cpu_fusion_80x60x32.npz: outputs of the reference's OWN CPU fusion
variant -- StereoMapper::outputFusionCPU (stereo_mapper.cpp:625-820) with transformMapCPU,
holeFillingCPU, depthPreditCPU, depthUpdateCPU, depthFuseCPU (:246-587) and the CASE 0 / CASE 1
argmin outputs (:628-706) -- compiled unmodified on the host by oracle/build_ref.py (build_cpu,
oracle/ref_cpu_unity.cpp with the stand-in headers of oracle/ref_stubs/).  Runs on the CPU of the
container that holds the reference sources; the fixture it writes travels with the tests.

Inputs, seeded: a 6-keyframe synthetic sequence at 80x60 (f = 64, 32 inverse-depth planes in
[0.1, 2.0] 1/m, 3 sources) mapped by the FP32 oracle (its cost volume, SGM volume and
winner-take-all depth); the WTA maps are then given a few values that exercise the masks of
:743-760 and :773-784 (depths above 10 and below 0.1; the oracle's own maps already hold the
1000 no-overlap marker and 0 rejections).  The two volumes are not stored: the tests rebuild
them with `inputs()` and check their SHA-256 digests, which the fixture keeps.  Recorded per
keyframe: the result of CASE >= 3 (the
fused depth; zeros for the first keyframe) and the propagation table of that step (p_table of
the step's current half), plus the final ping-pong state (alpha, beta, mu, sigma, both halves);
CASE 0 and CASE 1 results on the first keyframe's volumes.

  python tests/golden/make_ref_cpu_golden.py [--out PATH]
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

W, H, D, S, F, FOCAL, SEED = 80, 60, 32, 3, 6, 64.0, 404
OUT = os.path.join(HERE, f"ref_cpu_fusion_{W}x{H}x{D}.npz")


def load():
    from oracle import build_ref
    path = build_ref.build_cpu([(W, H, D)])[0]
    lib = ctypes.CDLL(path)
    fp, dp = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
    lib.refcpu_reset.argtypes = [dp, ctypes.c_float]
    lib.refcpu_output_fusion_cpu.argtypes = [ctypes.c_int, fp, fp, fp, dp, dp, ctypes.c_float, ctypes.c_float,
                                             ctypes.c_float, ctypes.c_float, fp, fp,
                                             ctypes.POINTER(ctypes.c_uint32)]
    w, h, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib.refcpu_shape(ctypes.byref(w), ctypes.byref(h), ctypes.byref(d))
    assert (w.value, h.value, d.value) == (W, H, D)
    return lib


def P(a, t=ctypes.c_float):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


def inputs():
    """Seeded sequence mapped by the FP32 oracle: per keyframe the WTA depth (with mask cases
    planted), the pose, and the first keyframe's cost and SGM volumes."""
    import oracle
    from probabilistic_mapping_b200 import scene
    seq = scene.make_sequence(W, H, FOCAL, S, F, seed=SEED)
    rho0, drho = scene.plane_range(D)
    p = oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=1 / 255, cost_mode=0, num_paths=8,
                      p1=0.003, p2=0.01, tau_so=3.5 / 255, uniqueness=0.95)
    rng = np.random.default_rng(SEED)
    wta, Rs, ts = [], [], []
    cost0 = sgm0 = None
    for k, fs in enumerate(seq):
        o = oracle.Mapper(p, fs.K, prec="f32")
        o.init_reference(fs.ref)
        for s in range(S):
            o.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        st = o.stages()
        d = st["depth"].astype(np.float32).copy()
        u = rng.uniform(size=d.shape)
        d[u < 0.02] = 15.0                       # > 10: zeroed before the fusion (:757-759)
        d[(u >= 0.02) & (u < 0.04)] = 0.05       # < 0.1: zeroed after it (:780-782)
        wta.append(d)
        Rs.append(np.asarray(fs.R_ref, np.float64))
        ts.append(np.asarray(fs.T_ref, np.float64).reshape(3))
        if k == 0:
            cost0, sgm0 = st["cost"].astype(np.float32), st["sgm"].astype(np.float32)
    K = seq[0].K
    return dict(wta=np.stack(wta), R=np.stack(Rs), t=np.stack(ts), K=np.asarray(K, np.float64),
                dep_sample=np.float32(drho), cost0=np.ascontiguousarray(cost0.reshape(-1)),
                sgm0=np.ascontiguousarray(sgm0.reshape(-1)))


def run_reference(lib, inp):
    N = W * H
    K = inp["K"]
    fx, fy, cx, cy = (np.float32(K[0, 0]), np.float32(K[1, 1]), np.float32(K[0, 2]), np.float32(K[1, 2]))
    out = {}
    # CASE 0 and CASE 1 on the first keyframe's volumes (the pose is not used there)
    for case, key in ((0, "case0"), (1, "case1")):
        assert lib.refcpu_reset(P(np.ascontiguousarray(K.reshape(-1)), ctypes.c_double), inp["dep_sample"]) == 0
        res = np.zeros(N, np.float32)
        st = lib.refcpu_output_fusion_cpu(case, P(inp["cost0"]), P(inp["sgm0"]), None,
                                          P(np.ascontiguousarray(inp["R"][0].reshape(-1)), ctypes.c_double),
                                          P(np.ascontiguousarray(inp["t"][0]), ctypes.c_double),
                                          fx, fy, cx, cy, P(res), None, None)
        assert st == 0
        out[key] = res.reshape(H, W)
    # CASE 3: the fusion sequence
    assert lib.refcpu_reset(P(np.ascontiguousarray(K.reshape(-1)), ctypes.c_double), inp["dep_sample"]) == 0
    results, tables = [], []
    state = np.zeros(8 * N, np.float32)
    table = np.zeros(2 * N, np.uint32)
    pre_index = 0
    for k in range(F):
        res = np.zeros(N, np.float32)
        st = lib.refcpu_output_fusion_cpu(3, None, None, P(np.ascontiguousarray(inp["wta"][k].reshape(-1))),
                                          P(np.ascontiguousarray(inp["R"][k].reshape(-1)), ctypes.c_double),
                                          P(np.ascontiguousarray(inp["t"][k]), ctypes.c_double),
                                          fx, fy, cx, cy, P(res), P(state), P(table, ctypes.c_uint32))
        assert st == 0
        results.append(res.reshape(H, W).copy())
        # the table of this step is the current half (pre_index ^ 1 before the swap); none on
        # the first keyframe
        tables.append(table.reshape(2, N)[pre_index ^ 1].copy() if k > 0 else np.zeros(N, np.uint32))
        if k > 0:
            pre_index ^= 1
    out["fused"] = np.stack(results)
    out["tables"] = np.stack(tables)
    out["state"] = state.reshape(4, 2, N)
    out["final_pre_index"] = np.int32(pre_index)
    return out


def main(path=OUT):
    lib = load()
    inp = inputs()
    out = run_reference(lib, inp)
    # the volumes are regenerated by the tests from the same seed (the FP32 oracle is
    # deterministic); the fixture keeps their digests instead of 1.2 MB of floats
    import hashlib
    data = {f"in_{k}": v for k, v in inp.items() if k not in ("cost0", "sgm0")}
    for k in ("cost0", "sgm0"):
        data[f"in_{k}_sha256"] = np.bytes_(hashlib.sha256(inp[k].tobytes()).hexdigest())
    data.update({f"ref_{k}": v for k, v in out.items()})
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({os.path.getsize(path)} bytes); fused pixels per keyframe:",
          [int((f != 0).sum()) for f in out["fused"]])


if __name__ == "__main__":
    main(sys.argv[sys.argv.index("--out") + 1] if "--out" in sys.argv else OUT)
