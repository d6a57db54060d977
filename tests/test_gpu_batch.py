"""The batched form against separate StereoMapper runs.

A batch of sequences with different shapes, precisions, samplers, path counts and cost modes (two
of them sharing one lane of cost/path volumes) is stepped over several keyframes; after every step each
sequence's fused depth and variance must equal, bit for bit, what a StereoMapper fed the same
frames and poses returns: the batch runs the same kernels, with the per-step values read from
device memory instead of kernel parameters.  With PM_BATCH_STATS, each sequence's pixel
counters must also equal the separate mapper's.
"""
import numpy as np
import pytest

from probabilistic_mapping_b200 import scene
from probabilistic_mapping_b200.batch import StereoBatch
from probabilistic_mapping_b200.mapper import StereoMapper

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

S = 3
COMMON = dict(intensity_scale=1 / 255, p1=0.003, p2=0.01, tau_so=3.5 / 255, uniqueness_ratio=0.95)
SEQS = [
    dict(width=96, height=64, num_planes=64, precision=0, cost_mode=0, num_paths=8),
    dict(width=128, height=96, num_planes=128, precision=1, cost_mode=1, num_paths=8),
    dict(width=96, height=64, num_planes=64, precision=0, cost_mode=0, num_paths=4),
    dict(width=96, height=64, num_planes=64, precision=0, cost_mode=0, num_paths=8),   # shares seq 0's lane
    dict(width=128, height=96, num_planes=64, precision=1, cost_mode=0, num_paths=8, sampler=2),  # FP32 texels
    dict(width=112, height=80, num_planes=64, precision=0, cost_mode=0, num_paths=8, sampler=2),  # FP32 form, texture
]


def make_configs():
    out = []
    for c in SEQS:
        rho0, _ = scene.plane_range(c["num_planes"])
        out.append(dict(c, rho0=rho0, **COMMON))
    return out


@pytest.mark.parametrize("host_io,autotune,priority,stats", [(True, False, False, False), (False, True, True, True)])
def test_batch_matches_separate_mappers(host_io, autotune, priority, stats):
    cfgs = make_configs()
    seqs = [scene.make_sequence(c["width"], c["height"], 0.8 * c["width"], S, 3, seed=50 + i)
            for i, c in enumerate(cfgs)]
    b = StereoBatch(cfgs, S, lanes=1, host_io=host_io, autotune=autotune, priority=priority, stats=stats)
    mappers = []
    for i, c in enumerate(cfgs):
        W, H, D = c["width"], c["height"], c["num_planes"]
        params = {k: v for k, v in c.items() if k not in ("width", "height", "num_planes")}
        m = StereoMapper(W, H, D, **params)
        _, drho = scene.plane_range(D)
        K = seqs[i][0].K
        m.initIntrinsic(K, 0.0, drho)
        if stats:
            m.enable_stats(True)
        b.init_intrinsic(i, K, drho)
        mappers.append(m)
    if autotune:
        for i in range(len(cfgs)):
            w, serial, ms = b.tuning(i)
            assert w in (2, 4, 8) and serial in (0, 1) and ms > 0
    nonzero = 0
    for step in range(3):
        for i, c in enumerate(cfgs):
            fs = seqs[i][step]
            frames = [fs.ref] + [fs.srcs[s] for s in range(S)]
            if not host_io:
                frames = [torch.from_numpy(np.ascontiguousarray(img)).cuda() for img in frames]
                torch.cuda.synchronize()   # the batch copies on its own stream
            for f, img in enumerate(frames):
                b.set_frame(i, f, img)
            b.set_poses(i, fs.R_ref, fs.T_ref, list(fs.R_srcs), list(fs.T_srcs))
        b.run()
        b.synchronize()
        for i, c in enumerate(cfgs):
            fs = seqs[i][step]
            m = mappers[i]
            m.initReference(fs.ref)
            for s in range(S):
                m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
            K = fs.K
            want_d, want_v = m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
            got_d, got_v = b.output(i) if host_io else b.copy_output(i)
            assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all(), (step, i)
            assert (got_v.view(np.uint32) == want_v.view(np.uint32)).all(), (step, i)
            nonzero += int((got_d != 0).sum() + (got_v != 0).sum())
            if stats:
                assert b.stats(i) == m.stats(), (step, i)
    assert nonzero > 0   # the fusion steps after the first keyframe produce depths and variances
    for m in mappers:
        m.close()
    b.close()


PERSIST_SEQS = [
    dict(width=96, height=64, num_planes=64, num_paths=8),
    dict(width=128, height=96, num_planes=128, num_paths=8),
    dict(width=112, height=80, num_planes=64, num_paths=4),
    dict(width=96, height=64, num_planes=64, num_paths=8),
    dict(width=160, height=120, num_planes=192, num_paths=8, tree_compat=1),   # planes left out of the tree
]


@pytest.mark.parametrize("precision,sampler,mode,stats", [(1, 2, 0, True), (0, 0, 0, True), (0, 2, 1, False),
                                                          (1, 0, 1, False)],
                         ids=["fp16-texture_f32-ref-stats", "fp32-exact-ref-stats", "fp32-texture_f32-corrected",
                              "fp16-exact-corrected"])
def test_persistent_batch_matches_separate_mappers(precision, sampler, mode, stats):
    """PM_BATCH_PERSISTENT: the cost tiles, rebases, SGM scanlines and combines of all sequences in
    one persistent launch give, bit for bit, what separate StereoMappers give (shapes, plane counts
    and path counts mixed; one precision, sampler and cost mode per batch)."""
    cfgs = []
    for c in PERSIST_SEQS:
        if precision == 1 and c["num_planes"] == 192:
            c = dict(c, num_planes=256)   # FP16 volumes need an even number of planes per lane
        rho0, _ = scene.plane_range(c["num_planes"])
        cfgs.append(dict(c, rho0=rho0, precision=precision, sampler=sampler, cost_mode=mode, **COMMON))
    seqs = [scene.make_sequence(c["width"], c["height"], 0.8 * c["width"], S, 3, seed=80 + i)
            for i, c in enumerate(cfgs)]
    b = StereoBatch(cfgs, S, lanes=0, host_io=True, persistent=True, stats=stats)
    mappers = []
    for i, c in enumerate(cfgs):
        params = {k: v for k, v in c.items() if k not in ("width", "height", "num_planes")}
        m = StereoMapper(c["width"], c["height"], c["num_planes"], **params)
        _, drho = scene.plane_range(c["num_planes"])
        m.initIntrinsic(seqs[i][0].K, 0.0, drho)
        if stats:
            m.enable_stats(True)
        b.init_intrinsic(i, seqs[i][0].K, drho)
        mappers.append(m)
    nonzero = 0
    for step in range(3):
        for i in range(len(cfgs)):
            fs = seqs[i][step]
            b.set_frame(i, 0, fs.ref)
            for s in range(S):
                b.set_frame(i, 1 + s, fs.srcs[s])
            b.set_poses(i, fs.R_ref, fs.T_ref, list(fs.R_srcs), list(fs.T_srcs))
        b.run()
        b.synchronize()
        for i in range(len(cfgs)):
            fs = seqs[i][step]
            m = mappers[i]
            m.initReference(fs.ref)
            for s in range(S):
                m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
            K = fs.K
            want_d, want_v = m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
            assert (b.wta_depth(i).view(np.uint32) == m.wta_depth().view(np.uint32)).all(), (step, i)
            got_d, got_v = b.output(i)
            assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all(), (step, i)
            assert (got_v.view(np.uint32) == want_v.view(np.uint32)).all(), (step, i)
            nonzero += int((got_d != 0).sum())
            if stats:
                assert b.stats(i) == m.stats(), (step, i)
    assert nonzero > 0
    for m in mappers:
        m.close()
    b.close()


def test_persistent_batch_rejects_what_it_cannot_schedule():
    from probabilistic_mapping_b200._lib import PmError
    rho0, _ = scene.plane_range(64)
    a = dict(width=96, height=64, num_planes=64, rho0=rho0, precision=0, **COMMON)
    with pytest.raises(PmError):   # one precision for all sequences
        StereoBatch([a, dict(a, precision=1)], S, persistent=True)
    with pytest.raises(PmError):   # every sequence with its own volumes
        StereoBatch([a, a], S, lanes=1, persistent=True)
    b = StereoBatch([a], S)
    with pytest.raises(PmError):   # counters only in a batch created with them
        b.stats(0)
    b.close()
