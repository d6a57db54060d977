"""Parity at the full-size configurations the benchmark times (640x480, f = 520, 128 inverse-depth
planes in [0.1, 2.0] 1/m, 5 sources, 8-path SGM, uniqueness 0.95, scaled intensities, reference
cost samples) -- the sizes where the long scanlines, the diagonal tails and the volume ordering
of the SGM kernels run at their real lengths.

 * Plain FP32 form (the drop-in StereoMapper): WTA depth and plane index bit-exact against the
   FP32 oracle; against the FP64 oracle WTA index identical on >= 99.5 % of the pixels and
   inverse-depth relative error <= 1 % where both hold a depth.
 * 30-keyframe fusion sequence (depth_fusion.cu:229-280 applied 29 times over the ping-pong state
   of stereo_mapper.cpp:237-241): every keyframe's WTA depth bit-exact against the FP32 oracle,
   fused depth and variance within 1e-4 relative (expf / rsqrtf differ by ulps from the host) on
   all but at most 1e-4 of the pixels per keyframe: the update's inlier test can land on the
   other side of its threshold for a pixel whose probability sits on it, and that pixel's state
   then follows the other branch for the rest of the sequence (measured: 1 of 307,200 pixels by
   keyframe 6).
 * The benchmark's batched FP16 form (texture unit on FP32 texels, autotuned SGM schedule, SGM at
   the greatest launch priority; 4 sequences of this shape in one pm_batch): WTA and fused outputs
   bit-exact against separate StereoMappers of the same form, and every sequence within the FP16
   form's bound (WTA index >= 99.5 %, inverse-depth error <= 1 %) against the FP64 transcription
   of the reference's own sampling -- tex2D with the texture unit's 8-bit interpolation weights
   (calc_cost.cu:93, 226-237), the oracle's bilinear_quant -- and within 1 % / 99 % of the FP64
   oracle with exact bilinear weights (measured 99.46-99.76 % on these four scenes: the 8-bit
   weights alone move a few tenths of a percent of the indices).

The seeds are the benchmark's own (bench.py: 1000 for the plain form, 2000 + i for the batch), so
these are the inputs the timed runs map.
"""
import json

import numpy as np
import pytest

import oracle
from probabilistic_mapping_b200 import _lib, scene
from probabilistic_mapping_b200.mapper import StereoMapper

pytestmark = pytest.mark.gpu

W, H, D, S, F_PX = 640, 480, 128, 5, 520.0
PATHS = 8
P1, P2, TAU, UNIQ = 0.003, 0.01, 3.5 / 255.0, 0.95


def mapper(precision=0, sampler=0):
    rho0, drho = scene.plane_range(D)
    m = StereoMapper(W, H, D, rho0=rho0, intensity_scale=1 / 255, num_paths=PATHS, p1=P1, p2=P2, tau_so=TAU,
                     uniqueness_ratio=UNIQ, cost_mode=0, precision=precision, sampler=sampler)
    return m, drho


def oracle_mapper(K, prec, quant=0):
    rho0, drho = scene.plane_range(D)
    return oracle.Mapper(oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=1 / 255, cost_mode=0,
                                       bilinear_quant=quant, num_paths=PATHS, p1=P1, p2=P2, tau_so=TAU,
                                       uniqueness=UNIQ), K, prec=prec)


def feed(obj, fs, oracle_side=False):
    if oracle_side:
        obj.init_reference(fs.ref)
    else:
        obj.initReference(fs.ref)
    for s in range(S):
        obj.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])


def has_depth(d):
    return (d > 0) & (d < 999)


def fp64_stats(depth, idx, d64, i64):
    both = has_depth(depth) & has_depth(d64)
    rel = np.abs(1.0 / depth[both].astype(np.float64) - 1.0 / d64[both]) * d64[both]
    return {"wta_index_match": float((idx == i64).mean()),
            "validity_match": float((has_depth(depth) == has_depth(d64)).mean()),
            "rel_inv_depth_median": float(np.median(rel)), "rel_inv_depth_p99": float(np.percentile(rel, 99)),
            "rel_inv_depth_max": float(rel.max()), "pixels_compared": int(both.sum())}


def test_plain_fp32_fullsize_against_fp32_and_fp64_oracles():
    fs = scene.make_sequence(W, H, F_PX, S, 1, seed=1000)[0]
    m, drho = mapper()
    m.initIntrinsic(fs.K, 0.0, drho)
    feed(m, fs)
    got = m.output()
    idx = m.wta_index()
    m.close()
    o32 = oracle_mapper(fs.K, "f32")
    feed(o32, fs, oracle_side=True)
    st = o32.stages()
    assert (got.view(np.uint32) == st["depth"].view(np.uint32)).all(), \
        f"{int((got.view(np.uint32) != st['depth'].view(np.uint32)).sum())} depths differ from the FP32 oracle"
    assert (idx == st["idx"]).all()
    o64 = oracle_mapper(fs.K, "f64")
    feed(o64, fs, oracle_side=True)
    s64 = o64.stages()
    r = fp64_stats(got, idx, s64["depth"], s64["idx"])
    print(json.dumps({"plain_fp32_vs_fp64": r}))
    assert r["wta_index_match"] >= 0.995
    assert r["rel_inv_depth_median"] <= 0.01 and r["rel_inv_depth_p99"] <= 0.01


def test_fusion_30_keyframes_fullsize_against_fp32_oracle():
    K_FRAMES = 30
    seq = scene.make_sequence(W, H, F_PX, S, K_FRAMES, seed=1000)
    K = seq[0].K
    fx, fy, cx, cy = K[0, 0], K[1, 1], K[0, 2], K[1, 2]
    m, drho = mapper()
    m.initIntrinsic(K, 0.0, drho)
    o = oracle_mapper(K, "f32")
    worst_d = worst_v = 0.0
    fused_px = diverged = 0
    for k, fs in enumerate(seq):
        feed(m, fs)
        feed(o, fs, oracle_side=True)
        got, var = m.outputFusion(fs.R_ref, fs.T_ref, fx, fy, cx, cy)
        st = o.output_fusion(fs.R_ref, fs.T_ref, fx, fy, cx, cy)
        assert (m.wta_depth().view(np.uint32) == st["depth"].view(np.uint32)).all(), f"keyframe {k}: WTA differs"
        if k == 0:
            assert (got == 0).all() and (var == 0).all()
            continue
        off_d = ~np.isclose(got, st["fused"], rtol=1e-4, atol=1e-5)
        off_v = ~np.isclose(var, st["variance"], rtol=1e-4, atol=1e-5)
        diverged = max(diverged, int(off_d.sum()), int(off_v.sum()))
        assert off_d.mean() <= 1e-4 and off_v.mean() <= 1e-4, \
            f"keyframe {k}: {int(off_d.sum())} fused depths, {int(off_v.sum())} variances beyond 1e-4"
        ok = ~(off_d | off_v)
        nz = (st["fused"] != 0) & ok
        fused_px += int(nz.sum())
        if nz.any():
            worst_d = max(worst_d, float(np.max(np.abs(got[nz] - st["fused"][nz]) / np.abs(st["fused"][nz]))))
        nv = (st["variance"] != 0) & ok
        if nv.any():
            worst_v = max(worst_v, float(np.max(np.abs(var[nv] - st["variance"][nv]) / np.abs(st["variance"][nv]))))
    m.close()
    print(json.dumps({"fusion_30_keyframes": {"max_rel_fused_depth": worst_d, "max_rel_variance": worst_v,
                                              "fused_pixels": fused_px, "most_diverged_pixels_in_a_keyframe": diverged}}))
    assert fused_px > 0


def test_batched_fp16_texture_fullsize_against_mappers_and_fp64():
    from probabilistic_mapping_b200.batch import StereoBatch
    B = 4
    rho0, drho = scene.plane_range(D)
    cfg = dict(width=W, height=H, num_planes=D, rho0=rho0, intensity_scale=1 / 255, num_paths=PATHS, p1=P1, p2=P2,
               tau_so=TAU, uniqueness_ratio=UNIQ, cost_mode=0, precision=_lib.PM_PREC_FP16,
               sampler=_lib.PM_SAMPLER_TEXTURE_F32)
    seqs = [scene.make_sequence(W, H, F_PX, S, 2, seed=2000 + i) for i in range(B)]
    b = StereoBatch([cfg] * B, S, lanes=0, host_io=True, autotune=True, priority=True)
    mappers = []
    for i in range(B):
        b.init_intrinsic(i, seqs[i][0].K, drho)
        m, _ = mapper(_lib.PM_PREC_FP16, _lib.PM_SAMPLER_TEXTURE_F32)
        m.initIntrinsic(seqs[i][0].K, 0.0, drho)
        mappers.append(m)
    report = []
    for step in range(2):
        for i in range(B):
            fs = seqs[i][step]
            b.set_frame(i, 0, fs.ref)
            for s in range(S):
                b.set_frame(i, 1 + s, fs.srcs[s])
            b.set_poses(i, fs.R_ref, fs.T_ref, list(fs.R_srcs), list(fs.T_srcs))
        b.run()
        b.synchronize()
        for i in range(B):
            fs = seqs[i][step]
            K = fs.K
            m = mappers[i]
            feed(m, fs)
            want_d, want_v = m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
            want_wta = m.wta_depth()
            got_d, got_v = b.output(i)
            got_wta = b.wta_depth(i)
            assert (got_wta.view(np.uint32) == want_wta.view(np.uint32)).all(), (step, i)
            assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all(), (step, i)
            assert (got_v.view(np.uint32) == want_v.view(np.uint32)).all(), (step, i)
            if step == 0:
                r = {}
                for quant in (1, 0):
                    o64 = oracle_mapper(K, "f64", quant)
                    feed(o64, fs, oracle_side=True)
                    s64 = o64.stages()
                    r["texture_weights" if quant else "exact_weights"] = fp64_stats(got_wta, m.wta_index(),
                                                                                    s64["depth"], s64["idx"])
                report.append(r)
                rq, re = r["texture_weights"], r["exact_weights"]
                assert rq["wta_index_match"] >= 0.995 and rq["rel_inv_depth_median"] <= 0.01, (i, r)
                assert re["wta_index_match"] >= 0.99 and re["rel_inv_depth_median"] <= 0.01, (i, r)
    print(json.dumps({"batched_fp16_texture_vs_fp64": report}))
    for m in mappers:
        m.close()
    b.close()
