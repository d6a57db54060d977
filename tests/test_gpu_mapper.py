"""StereoMapper drop-in (C ABI, host buffers) against the oracle's StereoMapper orchestration.

 * FP32 oracle (B200 op order): depth maps and WTA indices bit-exact.
 * FP64 oracle (line-for-line transcription): WTA plane index identical on >= 99.5% of the
   pixels, validity identical on >= 99.5%, depth within 1e-3 relative where both are valid.
 * Fusion over a keyframe sequence: fused depth / variance within 1e-4 relative of the FP32
   oracle (the update uses expf and rsqrtf).
"""
import numpy as np
import pytest

import oracle
from probabilistic_mapping_b200 import scene
from probabilistic_mapping_b200.mapper import StereoMapper

pytestmark = pytest.mark.gpu


def make(W, H, D, rho0, drho, mode, paths, uniq, K, scale=1 / 255):
    m = StereoMapper(W, H, D, rho0=rho0, intensity_scale=scale, num_paths=paths, p1=0.003, p2=0.01,
                     tau_so=3.5 / 255, uniqueness_ratio=uniq, cost_mode=mode)
    m.initIntrinsic(K, 0.0, drho)
    o = oracle.Mapper(oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=scale, cost_mode=mode,
                                    num_paths=paths, p1=0.003, p2=0.01, tau_so=3.5 / 255, uniqueness=uniq), K)
    return m, o


def feed(m, o, fs):
    m.initReference(fs.ref)
    o.init_reference(fs.ref)
    for s in range(fs.srcs.shape[0]):
        m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        o.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])


@pytest.mark.parametrize("mode,paths,D", [(0, 8, 64), (1, 8, 64), (0, 4, 128)])
def test_output_matches_fp32_oracle_bit_exact(mode, paths, D):
    W, H, S = 128, 96, 4
    fs = scene.make_frameset(W, H, 100.0, S, seed=11)
    rho0, drho = scene.plane_range(D)
    m, o = make(W, H, D, rho0, drho, mode, paths, 0.95, fs.K)
    o.prec = "f32"
    feed(m, o, fs)
    got = m.output()
    st = o.stages()
    for s in range(S):   # the kernels receive the FP64-composed homography rounded to float
        want_h = oracle.compose_homography(fs.K, fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s]).astype(np.float32)
        assert (m.homography(s) == want_h).all()
    assert (got.view(np.uint32) == st["depth"].view(np.uint32)).all()
    idx_host = m.wta_index()
    assert (idx_host == st["idx"]).all()
    m.close()


def test_output_against_fp64_oracle():
    W, H, D, S = 160, 120, 64, 4
    fs = scene.make_frameset(W, H, 130.0, S, seed=21)
    rho0, drho = scene.plane_range(D)
    m, o = make(W, H, D, rho0, drho, 0, 8, 0.95, fs.K)
    feed(m, o, fs)
    got = m.output()
    st = o.stages()
    want = st["depth"]
    valid_g = (got > 0) & (got < 999)
    valid_w = (want > 0) & (want < 999)
    assert (valid_g == valid_w).mean() >= 0.995
    assert ((got == 1000) == (want == 1000)).mean() >= 0.995
    both = valid_g & valid_w
    rel = np.abs(1 / got[both] - 1 / want[both]) * np.abs(want[both])
    assert np.median(rel) < 1e-5 and (rel < 1e-3).mean() >= 0.995
    m.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_fusion_sequence_matches_fp32_oracle(mode):
    W, H, D, S, F = 128, 96, 64, 3, 4
    seq = scene.make_sequence(W, H, 100.0, S, F, seed=31)
    rho0, drho = scene.plane_range(D)
    m, o = make(W, H, D, rho0, drho, mode, 8, 0.95, seq[0].K)
    o.prec = "f32"
    K = seq[0].K
    for k, fs in enumerate(seq):
        feed(m, o, fs)
        got, var = m.outputFusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
        st = o.output_fusion(fs.R_ref, fs.T_ref, K[0, 0], K[1, 1], K[0, 2], K[1, 2])
        assert (m.wta_depth().view(np.uint32) == st["depth"].view(np.uint32)).all()
        if k == 0:
            assert (got == 0).all() and (var == 0).all()
            continue
        np.testing.assert_allclose(got, st["fused"], rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(var, st["variance"], rtol=1e-4, atol=1e-5)
    a, b, mu, sg = m.get_state()
    assert np.isfinite(mu).all()
    m.close()


def test_pinned_and_device_inputs_match_host():
    import torch
    W, H, D, S = 96, 64, 64, 2
    fs = scene.make_frameset(W, H, 80.0, S, seed=41)
    rho0, drho = scene.plane_range(D)
    outs = []
    for kind in ("host", "pinned", "device"):
        m, _ = make(W, H, D, rho0, drho, 0, 8, 0.0, fs.K)
        conv = {"host": lambda a: a,
                "pinned": lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory(),
                "device": lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()}[kind]
        m.initReference(conv(fs.ref))
        for s in range(S):
            m.update(conv(fs.srcs[s]), fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        out = torch.empty((H, W), dtype=torch.float32, device="cuda") if kind == "device" else None
        r = m.output(out)
        torch.cuda.synchronize()
        outs.append(r.cpu().numpy() if kind == "device" else r)
        m.close()
    assert (outs[0] == outs[1]).all() and (outs[0] == outs[2]).all()


@pytest.mark.parametrize("precision,sampler", [(0, 0), (0, 2), (1, 0), (1, 1), (1, 2)],
                         ids=["fp32-exact", "fp32-texture_f32", "fp16-exact", "fp16-texture", "fp16-texture_f32"])
def test_source_overflow_folds_running_state(precision, sampler):
    """More update() calls than max_sources fold the queue into a running state; the result
    equals one pass over all sources.  FP32 forms: bit for bit (the texture samplers reuse source
    slots after the running state is written).  FP16 forms: the running state goes through the
    half volume and its per-pixel offset between the passes (unmeasured planes must stay
    negative there), so the bound is the FP16 form's: WTA plane index and validity identical on
    >= 99.5 % of the pixels, inverse depth within 1 % where both are valid."""
    W, H, D, S = 96, 64, 64, 5
    fs = scene.make_frameset(W, H, 80.0, S, seed=51)
    rho0, drho = scene.plane_range(D)
    res, idx = [], []
    for maxs in (16, 2):
        m = StereoMapper(W, H, D, rho0=rho0, intensity_scale=1 / 255, num_paths=4, p1=0.003, p2=0.01,
                         tau_so=3.5 / 255, max_sources=maxs, precision=precision, sampler=sampler)
        m.initIntrinsic(fs.K, 0.0, drho)
        m.initReference(fs.ref)
        for s in range(S):
            m.update(fs.srcs[s], fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
        res.append(m.output())
        idx.append(m.wta_index())
        m.close()
    if precision == 0:
        assert (res[0].view(np.uint32) == res[1].view(np.uint32)).all()
        assert (idx[0] == idx[1]).all()
        return
    assert (idx[0] == idx[1]).mean() >= 0.995
    valid = [(r > 0) & (r < 999) for r in res]
    assert (valid[0] == valid[1]).mean() >= 0.995
    both = valid[0] & valid[1]
    rel = np.abs(1 / res[0][both] - 1 / res[1][both]) * res[1][both]
    assert (rel <= 0.01).all()


def test_errors_are_reported_not_fatal():
    from probabilistic_mapping_b200._lib import PmError
    m = StereoMapper(64, 48, 64)
    with pytest.raises(PmError, match="initReference"):
        m.update(np.zeros((48, 64), np.uint8), np.eye(3), np.zeros(3), np.eye(3), np.zeros(3))
    with pytest.raises(PmError):
        m.output()
    m.initReference(np.zeros((48, 64), np.uint8))
    with pytest.raises(PmError, match="initIntrinsic"):
        m.update(np.zeros((48, 64), np.uint8), np.eye(3), np.zeros(3), np.eye(3), np.zeros(3))
    m.initIntrinsic(np.array([[50.0, 0, 32], [0, 50, 24], [0, 0, 1]]), 0.0, 0.03)
    bad = np.eye(3)
    bad[0, 0] = np.nan
    with pytest.raises(PmError, match="finite"):
        m.update(np.zeros((48, 64), np.uint8), bad, np.zeros(3), np.eye(3), np.zeros(3))
    # the handle stays usable
    m.update(np.zeros((48, 64), np.uint8), np.eye(3), np.zeros(3), np.eye(3), np.array([0.1, 0, 0]))
    out = m.output()
    assert out.shape == (48, 64)
    m.close()
