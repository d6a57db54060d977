"""Known-answer and property tests of the CPU oracle (runs without a GPU).

The reference tree holds no tests or fixtures, so the oracle is pinned here by cases whose
answer follows from the reference's code or from geometry, and by agreement between its FP64
and FP32 instantiations.
"""
import numpy as np
import pytest

import oracle
from conftest import homographies, small_case


def bitrev(v, bits):
    return int(format(v, f"0{bits}b")[::-1], 2)


@pytest.mark.parametrize("D", [32, 64, 128, 256])
def test_tree_order_power_of_two_is_bit_reversal(oracle_lib, D):
    """For power-of-two D the tie winner of filter_cost.cu:22-30 is the smallest bit-reversed index."""
    rank, incl = oracle.tree_order(D)
    assert incl.all()
    bits = D.bit_length() - 1
    order = sorted(range(D), key=lambda d: bitrev(d, bits))
    assert [int(np.where(rank == r)[0][0]) for r in range(D)] == order


def test_tree_order_non_power_of_two_drops_planes(oracle_lib):
    """D=192: the stride sequence 96,48,24,12,6,3,1 never folds slot 2 into slot 0 (sgm.cu:24-31)."""
    rank, incl = oracle.tree_order(192, 1)
    dropped = np.where(incl == 0)[0]
    assert len(dropped) > 0 and 2 in dropped
    # replay the reference loop literally and compare the surviving value
    rng = np.random.default_rng(0)
    for _ in range(20):
        c = rng.permutation(192).astype(np.float64)
        x = c.copy()
        i = 192 >> 1
        while i > 0:
            for d in range(i):
                if d + i < 192 and x[d + i] < x[d]:
                    x[d] = x[d + i]
            i >>= 1
        assert x[0] == c[incl == 1].min()
    rank0, incl0 = oracle.tree_order(192, 0)
    assert incl0.all()


def shifted_pair(W=64, H=40, disp=4, seed=0):
    rng = np.random.default_rng(seed)
    base = rng.uniform(0, 255, size=(H, W + 32))
    k = np.array([1, 4, 6, 4, 1], float)
    base = np.apply_along_axis(lambda r: np.convolve(r, k / k.sum(), "same"), 1, base)
    base = np.apply_along_axis(lambda r: np.convolve(r, k / k.sum(), "same"), 0, base)
    ref = np.clip(np.rint(base[:, 8:8 + W]), 0, 255).astype(np.uint8)
    src = np.clip(np.rint(base[:, 8 + disp:8 + disp + W]), 0, 255).astype(np.uint8)
    return ref, src


@pytest.mark.parametrize("mode", [0, 1])
def test_fronto_parallel_translation_selects_true_plane(oracle_lib, mode):
    """Camera translated by b along x (R = I): the source is the reference shifted by f*b*rho.
    A 4-pixel shift with f*b*drho = 0.5 px puts the true plane at index 8."""
    W, H, D = 64, 40, 32
    f, b = 50.0, 0.1
    drho = 0.5 / (f * b)
    ref, src = shifted_pair(W, H, 4)
    # +-1 intensity noise: a perfect match would make the aggregated minimum 0, which
    # filter_cost.cu:37-38 reports as non-overlap (DEP_INF)
    noise = np.random.default_rng(9).integers(-1, 2, size=src.shape)
    src = np.clip(src.astype(int) + noise, 0, 255).astype(np.uint8)
    K = np.array([[f, 0, W / 2], [0, f, H / 2], [0, 0, 1.0]])
    hom = oracle.compose_homography(K, np.eye(3), np.zeros(3), np.eye(3), np.array([b, 0, 0]))
    np.testing.assert_allclose(hom[:9], np.eye(3).reshape(-1), atol=1e-12)
    np.testing.assert_allclose(hom[9:], [-f * b, 0, 0], atol=1e-12)
    p = oracle.Params(W=W, H=H, D=D, drho=drho, cost_mode=mode)
    cost, cnt = oracle.calc_cost(p, ref, src[None], hom[None], "f64")
    interior = cost[2:-2, 8:-8]
    valid = (interior >= 0).all(axis=2)
    wta = np.argmin(np.where(interior < 0, np.inf, interior), axis=2)
    frac = (wta[valid] == 8).mean()
    assert frac > (0.99 if mode == 1 else 0.8)   # reference mode carries the bugged samples
    vol = oracle.sgm(p, ref, cost, "f64")
    depth, idx = oracle.filter_cost(p, vol, "f64")
    inner = depth[2:-2, 10:-10]
    good = (inner > 0) & (inner < 999)
    assert good.mean() > 0.8
    np.testing.assert_allclose(1 / inner[good], 8 * drho, rtol=0.05)


def test_identity_pose_gives_flat_cost_and_border_rejection(oracle_lib):
    """No baseline: every plane warps to the same place; the tree keeps plane 0 and
    filter_cost.cu:39-40 rejects it (depth 0)."""
    W, H, D = 32, 24, 32
    ref, _ = shifted_pair(W, H, 0)
    K = np.array([[30.0, 0, 16], [0, 30, 12], [0, 0, 1]])
    hom = oracle.compose_homography(K, np.eye(3), np.zeros(3), np.eye(3), np.zeros(3))
    p = oracle.Params(W=W, H=H, D=D, drho=0.05, cost_mode=1)
    cost, _ = oracle.calc_cost(p, ref, ref[None], hom[None], "f64")
    inner = cost[1:-1, 1:-1]
    assert (inner == inner[..., :1]).all()
    depth, idx = oracle.filter_cost(p, cost, "f64")
    assert (idx[1:-1, 1:-1] == 0).all()
    assert set(np.unique(depth[1:-1, 1:-1])) <= {0.0, 1000.0}


def test_sgm_is_bounded_below_by_paths_times_cost(oracle_lib):
    """Each path value is C + min(...) - min(L_prev) >= C, so the sum is >= P*C (sgm.cu:85-98)."""
    fs, p = small_case(W=48, H=32, D=32, S=2)
    cost, _ = oracle.calc_cost(p, fs.ref, fs.srcs, homographies(fs), "f64")
    vol = oracle.sgm(p, fs.ref, cost, "f64")
    valid = (cost >= 0).all(axis=2)
    assert valid.mean() > 0.5
    assert (vol[valid] >= p.num_paths * cost[valid] - 1e-12).all()
    assert (vol[~valid] == 0).all()   # COST_INF = 0 at pixels with an unmeasured plane


@pytest.mark.parametrize("paths", [4, 8])
def test_sgm_shifts_with_a_per_pixel_cost_shift(oracle_lib, paths):
    """The FP16 form stores C(p, .) - c_p and adds c_p back once per path: L_r(p, d) = C(p, d) +
    min(...) - min_k L_r(p - r, k) (sgm.cu:85-98) moves every L_r(p, .) by c_p when C(p, .) does,
    and the next pixel's min(...) and min_k terms move together, so the sum over P paths moves
    by exactly P c_p.  Checked on the FP64 transcription with a random shift at every valid
    pixel (invalid pixels, with a plane never measured, keep cost -1)."""
    fs, p = small_case(W=48, H=32, D=32, S=2)
    p.num_paths = paths
    cost, _ = oracle.calc_cost(p, fs.ref, fs.srcs, homographies(fs), "f64")
    valid = (cost >= 0).all(axis=2)
    shift = np.random.default_rng(3).random(valid.shape) * valid
    vol = oracle.sgm(p, fs.ref, cost, "f64")
    moved = oracle.sgm(p, fs.ref, np.where(valid[..., None], cost + shift[..., None], cost), "f64")
    np.testing.assert_allclose(moved, vol + paths * shift[..., None] * valid[..., None], rtol=0, atol=1e-9)
    # and so the winner-take-all index is unchanged
    _, i0 = oracle.filter_cost(p, vol, "f64")
    _, i1 = oracle.filter_cost(p, moved - paths * shift[..., None], "f64")
    assert (i0 == i1).mean() > 0.999


def test_fp32_and_fp64_instantiations_agree(oracle_lib):
    fs, p = small_case(W=96, H=64, D=64, S=3)
    homs = homographies(fs)
    res = {}
    for prec in ("f64", "f32"):
        cost, _ = oracle.calc_cost(p, fs.ref, fs.srcs, homs, prec)
        vol = oracle.sgm(p, fs.ref, cost, prec)
        res[prec] = oracle.filter_cost(p, vol, prec)
    d64, i64 = res["f64"]
    d32, i32 = res["f32"]
    assert (i64 == i32).mean() >= 0.995
    both = (d64 > 0) & (d64 < 999) & (d32 > 0) & (d32 < 999)
    assert np.median(np.abs(d64[both] - d32[both]) / d64[both]) < 1e-5


def vogiatzis(d, a, b, mu, s2, unc, outlier):
    """Closed form of the Gaussian x uniform update (depth_fusion.cu:189-216), in FP64."""
    S = unc + s2
    new_s2 = unc * s2 / S
    new_mu = (d * s2 + mu * unc) / S
    c1 = a / (a + b) * np.exp(-(d - mu) ** 2 / (2 * S)) / np.sqrt(2 * np.pi * S)
    c2 = b / (a + b) * outlier
    c1, c2 = c1 / (c1 + c2), c2 / (c1 + c2)
    f = c1 * (a + 1) / (a + b + 1) + c2 * a / (a + b + 1)
    e = c1 * (a + 1) * (a + 2) / ((a + b + 1) * (a + b + 2)) + c2 * a * (a + 1) / ((a + b + 1) * (a + b + 2))
    mu_p = c1 * new_mu + c2 * mu
    s2_p = c1 * (new_s2 + new_mu ** 2) + c2 * (s2 + mu ** 2) - mu_p ** 2
    a_p = (e - f) / (f - e / f)
    return a_p, a_p * (1 - f) / f, mu_p, s2_p


def test_fusion_update_closed_form(oracle_lib):
    """Identity motion: every confident pixel propagates onto itself and is updated with the
    closed-form Beta-Gaussian posterior; the output gate uses the pre-update inlier ratio."""
    W, H = 6, 5
    N = W * H
    pose = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32)
    cam = np.array([10, 10, 3, 2], np.float32)
    rng = np.random.default_rng(1)
    pre = oracle.FusionState(alpha=rng.uniform(5, 15, N), beta=rng.uniform(1, 5, N), mu=rng.uniform(1.5, 3, N),
                             sigma=rng.uniform(0.1, 1.0, N))
    cur = oracle.FusionState.zeros(W, H, np.float64)
    depth = pre.mu * rng.uniform(0.98, 1.02, N)
    mu0, s0 = pre.mu.copy(), pre.sigma.copy()
    a0, b0 = pre.alpha.copy(), pre.beta.copy()
    d_in = depth.copy()
    out, table = oracle.fuse_gpu(W, H, pose, cam, depth, pre, cur, "f64")
    for e in range(1, N):
        assert table[e] == e
        # transformMap moved mu (here in place: same depth) and inflated sigma by 0.05 * depth
        s_pred = s0[e] + 0.05 * pre.mu[e]
        want = vogiatzis(d_in[e], a0[e], b0[e], pre.mu[e], s_pred, 0.01 * d_in[e] ** 2, 1 / 50)
        np.testing.assert_allclose([cur.alpha[e], cur.beta[e], cur.mu[e], cur.sigma[e]], want, rtol=1e-5)
        gate = a0[e] / (a0[e] + b0[e]) > 0.6
        assert out[e] == (cur.mu[e] if gate else 0.0)
    # pixel 0 cannot be stored in the table (0 means empty); it takes its first occupied neighbour
    assert table[0] == W + 1


def test_fusion_initialises_new_pixels(oracle_lib):
    W, H = 4, 4
    pre = oracle.FusionState.zeros(W, H, np.float64)
    cur = oracle.FusionState.zeros(W, H, np.float64)
    depth = np.full(W * H, 2.0)
    depth[5] = 0.0
    pose = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32)
    out, table = oracle.fuse_gpu(W, H, pose, np.array([5, 5, 2, 2], np.float32), depth, pre, cur, "f64")
    assert (table == 0).all()
    init = np.arange(W * H) != 5
    assert (cur.alpha[init] == 10).all() and (cur.beta[init] == 10).all() and (cur.sigma[init] == 2500).all()
    assert (out[init] == 2.0).all() and out[5] == 0.0 and cur.alpha[5] == -1.0   # depth_fusion.cu:129,161-174


def cpu_state(W, H, pixels):
    N = W * H
    st = {k: np.zeros((2, N), np.float32) for k in ("alpha", "beta", "mu", "sigma")}
    st["table"] = np.zeros((2, N), np.uint32)
    for i, dep in pixels:
        st["alpha"][0, i], st["beta"][0, i], st["mu"][0, i], st["sigma"][0, i] = 10, 1, dep, 1.0
    return st


def test_cpu_fusion_variant_sequential_z_test(oracle_lib):
    """transformMapCPU compares the occupant's moved depth with the candidate's unmoved depth
    and, when the candidate wins, writes the candidate's depth into the occupant's mu
    (stereo_mapper.cpp:311-324); raster order decides who is the occupant."""
    W, H, f = 8, 8, 10.0
    cam = np.array([f, f, 4, 4], np.float32)

    def pose(tx):
        p = np.zeros(12)
        p[[0, 4, 8]] = 1
        p[9] = tx
        return p

    # pixels 9 (x=1, depth 1) and 10 (x=2, depth 2) land on cell (3, 1); the occupant (9) is nearer
    st = cpu_state(W, H, [(9, 1.0), (10, 2.0)])
    oracle.fuse_cpu(W, H, pose(0.2), cam, 0, np.full(W * H, 3.0, np.float32), st)
    assert st["table"][1][11] == (1 << 16) | 1
    assert st["mu"][0][9] == 1.0 and st["mu"][0][10] == 2.0
    # pixels 9 (depth 2) and 10 (depth 1) land on cell (0, 1); the later, nearer candidate takes the
    # cell and overwrites the occupant's mu with its own depth
    st = cpu_state(W, H, [(9, 2.0), (10, 1.0)])
    oracle.fuse_cpu(W, H, pose(-0.2), cam, 0, np.full(W * H, 3.0, np.float32), st)
    assert st["table"][1][8] == (1 << 16) | 2
    assert st["mu"][0][9] == 1.0
    # 7x7 hole filling spreads the occupant from interior cells only (x, y in [3, H-3))
    assert (st["table"][1] == 0).sum() > 0


def test_convert_round_trip(oracle_lib):
    W, H, pitch = 5, 3, 32
    lin = np.arange(W * H, dtype=np.float32)
    pitched = oracle.convert(W, H, lin, 1, pitch)
    back = oracle.convert(W, H, pitched, 0, pitch)
    assert (back == lin).all()
    rows = pitched.reshape(H, pitch)[:, :4 * W].copy().view(np.float32)
    assert (rows.reshape(-1) == lin).all()


def test_homography_matches_formula(oracle_lib):
    rng = np.random.default_rng(3)
    from probabilistic_mapping_b200.scene import rodrigues
    K = np.array([[500.0, 0, 320], [0, -480, 240], [0, 0, 1]])   # negative fy as in evaluate.cc:38
    Rl = rodrigues(rng.normal(size=3), 0.2)
    Rr = rodrigues(rng.normal(size=3), 0.3)
    Tl, Tr = rng.normal(size=3), rng.normal(size=3)
    h = oracle.compose_homography(K, Rl, Tl, Rr, Tr)
    H1 = K @ Rr.T @ Rl @ np.linalg.inv(K)
    H2 = K @ Rr.T @ (Tl - Tr)
    np.testing.assert_allclose(h[:9], H1.reshape(-1), rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(h[9:], H2, rtol=1e-12, atol=1e-9)
