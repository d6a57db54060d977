"""Stage-level parity of the CUDA kernels against the CPU oracle, through the C ABI.

Bit-exact: cost volume, SGM sums, winner-take-all index and depth, against the oracle's FP32
instantiation (same operation order).  The fusion stage uses CUDA's expf/rsqrtf, so its
floating-point outputs are compared with a stated tolerance and its integer table exactly.
"""
import ctypes

import numpy as np
import pytest

import oracle
from conftest import homographies, small_case

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def config(p, precision=0):
    from probabilistic_mapping_b200 import _lib
    c = _lib.default_config(p.W, p.H, p.D)
    c.rho0, c.rho_step, c.intensity_scale = p.rho0, p.drho, p.intensity_scale
    c.num_paths = p.num_paths
    c.p1, c.p2, c.tau_so, c.q1, c.q2 = p.p1, p.p2, p.tau_so, p.q1, p.q2
    c.var_scale, c.uniqueness_ratio = p.var_scale, p.uniqueness
    c.cost_mode, c.tree_compat, c.precision = p.cost_mode, p.tree_compat, precision
    return c


def upload_images(lib, fs, scale):
    H, W = fs.ref.shape
    S = fs.srcs.shape[0]
    dev = torch.device("cuda")
    r8 = torch.from_numpy(fs.ref).to(dev)
    s8 = torch.from_numpy(np.ascontiguousarray(fs.srcs)).to(dev)
    rf = torch.empty((H, W), dtype=torch.float32, device=dev)
    sf = torch.empty((S, H, W), dtype=torch.float32, device=dev)
    assert lib.pm_stage_to_float(W, H, vp(r8), W, vp(rf), scale, None) == 0
    for s in range(S):
        assert lib.pm_stage_to_float(W, H, vp(s8[s]), W, vp(sf[s]), scale, None) == 0
    return rf, sf


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


@pytest.mark.parametrize("mode", [0, 1])
def test_calc_cost_bit_exact(pm_lib, mode):
    fs, p = small_case(mode=mode)
    homs = homographies(fs)
    want_cost, want_cnt = oracle.calc_cost(p, fs.ref, fs.srcs, homs, "f32")
    rf, sf = upload_images(pm_lib, fs, p.intensity_scale)
    cost = torch.empty((p.H, p.W, p.D), dtype=torch.float32, device="cuda")
    inv = torch.empty((p.H, p.W), dtype=torch.uint8, device="cuda")
    hf = np.ascontiguousarray(homs, np.float32).reshape(-1)
    cfg = config(p)
    st = pm_lib.pm_stage_calc_cost(ctypes.byref(cfg), vp(rf), vp(sf), fs.srcs.shape[0], fptr(hf), vp(cost),
                                   None, vp(inv), None)
    assert st == 0
    torch.cuda.synchronize()
    got = cost.cpu().numpy()
    assert (bits(got) == bits(want_cost)).all(), np.abs(got - want_cost).max()
    assert (inv.cpu().numpy().astype(bool) == (want_cnt == 0).any(axis=2)).all()
    # both outcomes of the voxel test occur in this scene
    assert (want_cost < 0).any() and (want_cost >= 0).any()


def test_calc_cost_incremental_matches_single_pass(pm_lib):
    """Folding sources over several calls (the reference's per-update running mean) equals
    folding them in one pass."""
    fs, p = small_case(S=4)
    homs = homographies(fs)
    want_cost, want_cnt = oracle.calc_cost(p, fs.ref, fs.srcs, homs, "f32")
    rf, sf = upload_images(pm_lib, fs, p.intensity_scale)
    cost = torch.full((p.H, p.W, p.D), -1.0, dtype=torch.float32, device="cuda")
    cnt = torch.zeros((p.H, p.W, p.D), dtype=torch.float32, device="cuda")
    hf = np.ascontiguousarray(homs, np.float32).reshape(-1)
    cfg = config(p)
    for a, b in ((0, 1), (1, 3), (3, 4)):
        st = pm_lib.pm_stage_calc_cost(ctypes.byref(cfg), vp(rf), vp(sf[a]), b - a, fptr(hf[12 * a:]),
                                       vp(cost), vp(cnt), None, None)
        assert st == 0
    torch.cuda.synchronize()
    assert (bits(cost.cpu().numpy()) == bits(want_cost)).all()
    assert (cnt.cpu().numpy() == want_cnt).all()


@pytest.mark.parametrize("offset", [1, 2])
def test_calc_cost_unaligned_buffers(pm_lib, offset):
    """Volume and count buffers that start 4 or 8 bytes past a 16-byte boundary (the kernel's
    vector stores need 16): the same values as the oracle, through element stores."""
    fs, p = small_case(S=3)
    homs = homographies(fs)
    want_cost, want_cnt = oracle.calc_cost(p, fs.ref, fs.srcs, homs, "f32")
    rf, sf = upload_images(pm_lib, fs, p.intensity_scale)
    V = p.H * p.W * p.D
    cbuf = torch.full((V + 4,), 7.0, dtype=torch.float32, device="cuda")
    nbuf = torch.full((V + 4,), 7.0, dtype=torch.float32, device="cuda")
    cost, cnt = cbuf[offset:offset + V], nbuf[offset:offset + V]
    assert cost.data_ptr() % 16 and cnt.data_ptr() % 16
    hf = np.ascontiguousarray(homs, np.float32).reshape(-1)
    cfg = config(p)
    # a first pass without counts, then the rest folded into it with counts
    st = pm_lib.pm_stage_calc_cost(ctypes.byref(cfg), vp(rf), vp(sf), 3, fptr(hf), vp(cost), None, None, None)
    assert st == 0
    torch.cuda.synchronize()
    assert (bits(cost.cpu().numpy()) == bits(want_cost.reshape(-1))).all()
    cost.fill_(-1.0)
    cnt.zero_()
    for a, b in ((0, 2), (2, 3)):
        st = pm_lib.pm_stage_calc_cost(ctypes.byref(cfg), vp(rf), vp(sf[a]), b - a, fptr(hf[12 * a:]),
                                       vp(cost), vp(cnt), None, None)
        assert st == 0
    torch.cuda.synchronize()
    assert (bits(cost.cpu().numpy()) == bits(want_cost.reshape(-1))).all()
    assert (cnt.cpu().numpy() == want_cnt.reshape(-1)).all()
    # nothing outside the views was written
    for buf in (cbuf, nbuf):
        h = buf.cpu().numpy()
        assert (h[:offset] == 7.0).all() and (h[offset + V:] == 7.0).all()


@pytest.mark.parametrize("D,paths,compat,uniq", [(64, 8, 1, 0.95), (64, 4, 1, 0.0), (96, 8, 1, 0.95),
                                                 (96, 4, 0, 0.0), (128, 8, 1, 0.95), (192, 4, 1, 0.0)])
def test_sgm_and_filter_bit_exact(pm_lib, D, paths, compat, uniq):
    fs, p = small_case(D=D, paths=paths, uniq=uniq, W=80, H=56)
    p.tree_compat = compat
    homs = homographies(fs)
    cost, _ = oracle.calc_cost(p, fs.ref, fs.srcs, homs, "f32")
    want_sum = oracle.sgm(p, fs.ref, cost, "f32")
    want_depth, want_idx = oracle.filter_cost(p, want_sum, "f32")
    rf, _ = upload_images(pm_lib, fs, p.intensity_scale)
    dcost = torch.from_numpy(cost).cuda()
    out = torch.empty_like(dcost)
    # the documented minimum scratch (num_paths/2 - 1 pair volumes) followed by a guard volume
    npairs = p.num_paths // 2
    part = torch.full((npairs,) + tuple(dcost.shape), 7.0, dtype=torch.float32, device="cuda")
    cfg = config(p)
    assert pm_lib.pm_stage_sgm(ctypes.byref(cfg), vp(dcost), vp(rf), vp(out), vp(part), None) == 0
    torch.cuda.synchronize()
    assert (part[npairs - 1] == 7.0).all(), "pm_stage_sgm wrote past its scratch"
    depth = torch.empty((p.H, p.W), dtype=torch.float32, device="cuda")
    idx = torch.empty((p.H, p.W), dtype=torch.int32, device="cuda")
    assert pm_lib.pm_stage_filter(ctypes.byref(cfg), vp(out), vp(depth), 4 * p.W, vp(idx), None) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert (bits(got) == bits(want_sum)).all(), np.abs(got - want_sum).max()
    assert (idx.cpu().numpy() == want_idx).all()
    assert (bits(depth.cpu().numpy()) == bits(want_depth)).all()
    # the reference's sequential path order differs only by rounding
    p.sum_order = 0
    seq_sum = oracle.sgm(p, fs.ref, cost, "f32")
    p.sum_order = 1
    np.testing.assert_allclose(seq_sum, want_sum, rtol=2e-6, atol=1e-6)
    # fused last path + filter gives the same depth and index
    scratch = torch.full((npairs + 1,) + tuple(dcost.shape), 7.0, dtype=torch.float32, device="cuda")
    depth2 = torch.zeros((p.H, p.W + 3), dtype=torch.float32, device="cuda")   # pitched output
    idx2 = torch.empty((p.H, p.W), dtype=torch.int32, device="cuda")
    assert pm_lib.pm_stage_sgm_filter(ctypes.byref(cfg), vp(dcost), vp(rf), vp(scratch), vp(depth2),
                                      4 * (p.W + 3), vp(idx2), None) == 0
    torch.cuda.synchronize()
    assert (idx2.cpu().numpy() == want_idx).all()
    assert (bits(depth2.cpu().numpy()[:, :p.W]) == bits(want_depth)).all()
    assert (scratch[npairs] == 7.0).all(), "pm_stage_sgm_filter wrote past its scratch"
    # every decision branch of filter_cost.cu:37-52 is exercised
    assert (want_depth == 1000.0).any() and (want_depth == 0).any() and ((want_depth > 0) & (want_depth < 1000)).any()


def test_filter_tie_break_follows_reduction_tree(pm_lib):
    """Equal minima: the winner is the one the reference's tree reduction keeps."""
    W, H, D = 32, 4, 64
    p = oracle.Params(W=W, H=H, D=D, drho=0.03, num_paths=4)
    rng = np.random.default_rng(0)
    vol = rng.uniform(1.0, 2.0, size=(H, W, D)).astype(np.float32)
    for x in range(W):
        for y in range(H):
            ties = rng.choice(D, size=rng.integers(2, 6), replace=False)
            vol[y, x, ties] = 0.5
    vol[0, 0, :] = 0.7   # an all-equal pixel
    want_depth, want_idx = oracle.filter_cost(p, vol, "f32")
    rank, _ = oracle.tree_order(D)
    assert (rank[want_idx[0, 0]] == 0)
    dvol = torch.from_numpy(vol).cuda()
    depth = torch.empty((H, W), dtype=torch.float32, device="cuda")
    idx = torch.empty((H, W), dtype=torch.int32, device="cuda")
    cfg = config(p)
    assert pm_lib.pm_stage_filter(ctypes.byref(cfg), vp(dvol), vp(depth), 4 * W, vp(idx), None) == 0
    torch.cuda.synchronize()
    assert (idx.cpu().numpy() == want_idx).all()
    assert (bits(depth.cpu().numpy()) == bits(want_depth)).all()


def fusion_inputs(seed=5, W=96, H=64):
    """A realistic previous state (from one oracle frame) and the next frame's WTA depth."""
    from probabilistic_mapping_b200 import scene
    seq = scene.make_sequence(W, H, 0.8 * W, 2, 2, seed=seed)
    rng = np.random.default_rng(seed)
    N = W * H
    d0 = seq[0].gt_depth.reshape(-1).astype(np.float32)
    pre = oracle.FusionState(
        alpha=rng.uniform(0.0, 20.0, N).astype(np.float32),
        beta=rng.uniform(0.5, 12.0, N).astype(np.float32),
        mu=(d0 * rng.uniform(0.97, 1.03, N)).astype(np.float32),
        sigma=rng.uniform(0.01, 3.0, N).astype(np.float32))
    pre.alpha[rng.uniform(size=N) < 0.1] = 0.0
    depth = (seq[1].gt_depth.reshape(-1) * rng.uniform(0.95, 1.05, N)).astype(np.float32)
    depth[rng.uniform(size=N) < 0.1] = 0.0
    depth[rng.uniform(size=N) < 0.02] = 1000.0
    rel = oracle.relative_pose(seq[1].R_ref, seq[1].T_ref, seq[0].R_ref, seq[0].T_ref).astype(np.float32)
    K = seq[0].K
    cam = np.array([K[0, 0], K[1, 1], K[0, 2], K[1, 2]], np.float32)
    return W, H, rel, cam, depth, pre


def test_depth_fuse_against_oracle(pm_lib):
    W, H, rel, cam, depth, pre = fusion_inputs()
    N = W * H
    cur = oracle.FusionState(*[np.full(N, 7.0, np.float32) for _ in range(4)])
    d_pre = [torch.from_numpy(a.copy()).cuda() for a in (pre.alpha, pre.beta, pre.mu, pre.sigma)]
    d_cur = [torch.from_numpy(a.copy()).cuda() for a in (cur.alpha, cur.beta, cur.mu, cur.sigma)]
    d_depth = torch.from_numpy(depth.copy()).cuda()
    zt = torch.empty(N, dtype=torch.int64, device="cuda")
    table = torch.empty(N, dtype=torch.int32, device="cuda")
    want_depth, want_table = oracle.fuse_gpu(W, H, rel, cam, depth.copy(), pre, cur, "f32")
    prep = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in d_pre])
    curp = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in d_cur])
    st = pm_lib.pm_stage_depth_fuse(W, H, fptr(rel), fptr(cam), vp(d_depth), prep, curp, vp(zt), vp(table), None)
    assert st == 0
    torch.cuda.synchronize()
    assert (table.cpu().numpy() == want_table).all()
    assert (want_table != 0).mean() > 0.5
    # transformMap's in-place edits of the previous state are bit-exact (no transcendental)
    for got, want in zip(d_pre, (pre.alpha, pre.beta, pre.mu, pre.sigma)):
        assert (bits(got.cpu().numpy()) == bits(want)).all()
    # depthUpdate uses expf/rsqrtf: tolerance 1e-4 relative
    for got, want in zip(d_cur + [d_depth], (cur.alpha, cur.beta, cur.mu, cur.sigma, want_depth)):
        g = got.cpu().numpy()
        np.testing.assert_allclose(g, want, rtol=1e-4, atol=1e-5)


def test_convert_round_trip(pm_lib):
    W, H = 37, 11
    pitch = 4 * W + 52
    lin = torch.arange(W * H, dtype=torch.float32, device="cuda")
    pitched = torch.zeros(H * pitch // 4, dtype=torch.float32, device="cuda")
    back = torch.zeros(W * H, dtype=torch.float32, device="cuda")
    assert pm_lib.pm_stage_convert(W, H, vp(lin), vp(pitched), 1, pitch, None) == 0
    assert pm_lib.pm_stage_convert(W, H, vp(pitched), vp(back), 0, pitch, None) == 0
    torch.cuda.synchronize()
    want = oracle.convert(W, H, lin.cpu().numpy(), 1, pitch)
    assert (pitched.cpu().numpy().view(np.uint8) == want).all()
    assert (back == lin).all()
