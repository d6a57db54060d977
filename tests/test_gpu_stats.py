"""pm_stats pixel counters on the GPU against the FP32 oracle's classes, over keyframe sequences.

The winner-take-all classes come from bit-exact maps, so they must match the oracle exactly on
every frame.  The fusion counters match exactly up to the first Bayesian update (the state it
starts from is exact); later steps start from states that differ from the oracle's in the last
bits (CUDA's expf against the host's), so a threshold test may flip on a few pixels there.
Turning the counters on must not change any output bit.
"""
import numpy as np
import pytest

import oracle
from probabilistic_mapping_b200 import _lib, scene
from probabilistic_mapping_b200._lib import PmError
from probabilistic_mapping_b200.mapper import StereoMapper

pytestmark = pytest.mark.gpu


def prm(D, mode=0, **kw):
    rho0, _ = scene.plane_range(D)
    p = dict(rho0=rho0, intensity_scale=1 / 255, num_paths=8, p1=0.003, p2=0.01, tau_so=3.5 / 255,
             uniqueness_ratio=0.95, cost_mode=mode)
    p.update(kw)
    return p


def feed(m, fs, o=None):
    m.initReference(fs.ref)
    if o is not None:
        o.init_reference(fs.ref)
    for s in range(fs.srcs.shape[0]):
        m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        if o is not None:
            o.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])


@pytest.mark.parametrize("variant", ["gpu_fusion", "cpu_fusion"])
def test_counters_match_fp32_oracle(variant):
    W, H, D, S, F = 128, 96, 64, 3, 5
    seq = scene.make_sequence(W, H, 100.0, S, F, seed=71)
    rho0, drho = scene.plane_range(D)
    fv = _lib.PM_FUSION_CPU_PATH if variant == "cpu_fusion" else _lib.PM_FUSION_GPU
    m = StereoMapper(W, H, D, fusion_variant=fv, **prm(D))
    K = seq[0].K
    m.initIntrinsic(K, 0.0, drho)
    m.enable_stats(True)
    o = oracle.Mapper(oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=1 / 255, num_paths=8,
                                    p1=0.003, p2=0.01, tau_so=3.5 / 255, uniqueness=0.95), K, prec="f32",
                      fusion="cpu" if variant == "cpu_fusion" else "gpu")
    N = W * H
    for k, fs in enumerate(seq):
        feed(m, fs, o)
        m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
        want = o.output_fusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])["stats"]
        got = m.stats()
        for n in oracle.WTA_CLASSES:
            assert got[n] == want[n], (k, n, got[n], want[n])
        for n in oracle.FUSION_COUNTS:
            if k <= 2:
                assert got[n] == want[n], (k, n, got[n], want[n])
            else:
                assert abs(got[n] - want[n]) <= max(2, N // 1000), (k, n, got[n], want[n])
        if k > 0:
            assert sum(got[n] for n in oracle.FUSION_COUNTS[:5]) == N
            assert got["pred_none"] + got["pred_copied"] == N
            assert sum(got[n] for n in oracle.FUSION_COUNTS[8:]) == N
    m.close()


@pytest.mark.parametrize("precision,sampler", [(0, 0), (1, 2)])
def test_counters_leave_outputs_unchanged(precision, sampler):
    W, H, D, S, F = 160, 120, 64, 3, 3
    seq = scene.make_sequence(W, H, 130.0, S, F, seed=73)
    _, drho = scene.plane_range(D)
    K = seq[0].K
    outs = []
    for on in (False, True):
        m = StereoMapper(W, H, D, precision=precision, sampler=sampler, **prm(D))
        m.initIntrinsic(K, 0.0, drho)
        if on:
            m.enable_stats(True)
        res = []
        for fs in seq:
            feed(m, fs)
            d, v = m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
            res += [m.wta_depth().copy(), m.wta_index().copy(), d.copy(), v.copy()]
        if on:
            st = m.stats()
            assert sum(st[n] for n in oracle.WTA_CLASSES) == W * H
        outs.append(res)
        m.close()
    for a, b in zip(*outs):
        assert (a.view(np.uint32) == b.view(np.uint32)).all()


def test_counters_per_call_and_off_state():
    W, H, D, S = 96, 64, 64, 2
    fs = scene.make_frameset(W, H, 80.0, S, seed=75)
    rho0, drho = scene.plane_range(D)
    m = StereoMapper(W, H, D, **prm(D))
    m.initIntrinsic(fs.K, 0.0, drho)
    with pytest.raises(PmError) as e:
        m.stats()
    assert e.value.status == _lib.PM_ERR_BAD_STATE
    m.enable_stats(True)
    feed(m, fs)
    depth = m.output()
    st = m.stats()
    assert st["wta_no_overlap"] == int(np.count_nonzero(depth == 1000.0))
    assert st["wta_depth"] == int(np.count_nonzero((depth > 0) & (depth != 1000.0)))
    assert sum(st[n] for n in oracle.WTA_CLASSES) == W * H
    assert all(st[n] == 0 for n in oracle.FUSION_COUNTS)   # pm_output runs no fusion
    st2 = m.stats()
    assert st2 == st
    m.outputCase(1)   # the debug argmin is not a winner-take-all filter: counters restart at zero
    assert all(v == 0 for v in m.stats().values())
    m.enable_stats(False)
    with pytest.raises(PmError):
        m.stats()
    m.close()
