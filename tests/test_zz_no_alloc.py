"""pm_stage_depth_fuse_noalloc: the depth-fusion step for callers that cannot allocate device
memory while they run (a flight-control loop, a host framework that owns every device buffer,
work recorded into a CUDA graph).  It keeps its z-buffer in a library-owned device array instead
of a caller buffer.  Two calls in a row, on different inputs, must give exactly what the
allocating entry point gives, so nothing leaks between calls through the shared array.

This file is named to be collected last: if it fails, a run that stops at the first failure
has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def inputs(seed, W=96, H=64):
    """A previous-keyframe state and the next WTA depth map, from a seeded synthetic scene."""
    import oracle
    from probabilistic_mapping_b200 import scene
    seq = scene.make_sequence(W, H, 0.8 * W, 1, 2, seed=seed)
    rng = np.random.default_rng(seed)
    N = W * H
    d0 = seq[0].gt_depth.reshape(-1).astype(np.float32)
    state = [rng.uniform(0.0, 20.0, N), rng.uniform(0.5, 12.0, N), d0 * rng.uniform(0.97, 1.03, N),
             rng.uniform(0.01, 3.0, N)]
    state = [s.astype(np.float32) for s in state]
    state[0][rng.uniform(size=N) < 0.1] = 0.0
    depth = (seq[1].gt_depth.reshape(-1) * rng.uniform(0.95, 1.05, N)).astype(np.float32)
    depth[rng.uniform(size=N) < 0.1] = 0.0
    pose = oracle.relative_pose(seq[1].R_ref, seq[1].T_ref, seq[0].R_ref, seq[0].T_ref).astype(np.float32)
    K = seq[0].K
    cam = np.array([K[0, 0], K[1, 1], K[0, 2], K[1, 2]], np.float32)
    return W, H, pose, cam, depth, state


def run(lib, case, noalloc):
    W, H, pose, cam, depth, state = case
    N = W * H
    pre = [torch.from_numpy(s.copy()).cuda() for s in state]
    cur = [torch.full((N,), 3.0, dtype=torch.float32, device="cuda") for _ in range(4)]
    d = torch.from_numpy(depth.copy()).cuda()
    table = torch.empty(N, dtype=torch.int32, device="cuda")
    prep = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in pre])
    curp = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in cur])
    if noalloc:
        st = lib.pm_stage_depth_fuse_noalloc(W, H, fptr(pose), fptr(cam), vp(d), prep, curp, vp(table), None)
    else:
        zt = torch.empty(N, dtype=torch.int64, device="cuda")
        st = lib.pm_stage_depth_fuse(W, H, fptr(pose), fptr(cam), vp(d), prep, curp, vp(zt), vp(table), None)
    assert st == 0
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in [d, table] + pre + cur]


def test_noalloc_fusion_matches_allocating_entry_point_twice(pm_lib):
    # two calls in a row on different scenes and poses; the first image is the larger one, so
    # the second call runs over an array that still holds the first call's z-buffer beyond its
    # own pixels.  Both entry points run the same kernels on the same inputs: bit-identical.
    for seed, (W, H) in ((5, (128, 96)), (6, (96, 64))):
        case = inputs(seed, W, H)
        want = run(pm_lib, case, noalloc=False)
        got = run(pm_lib, case, noalloc=True)
        assert (got[1] == want[1]).all(), "propagation tables differ"
        assert (want[1] != 0).mean() > 0.5
        for g, w in zip(got[:1] + got[2:], want[:1] + want[2:]):
            assert (g.view(np.uint32) == w.view(np.uint32)).all(), "fusion outputs differ"


def test_noalloc_rejects_a_stream_of_another_context(pm_lib):
    # a stream created in a context other than the current one: the array address would be the
    # wrong context's, so the call refuses it before any GPU work
    import ctypes.util
    cu = ctypes.CDLL(ctypes.util.find_library("cuda") or "libcuda.so.1")
    torch.cuda.init()
    dev = ctypes.c_int(0)
    assert cu.cuDeviceGet(ctypes.byref(dev), torch.cuda.current_device()) == 0
    ctx = ctypes.c_void_p()
    assert cu.cuCtxCreate_v2(ctypes.byref(ctx), 0, dev) == 0   # made current by the call
    try:
        stream = ctypes.c_void_p()
        assert cu.cuStreamCreate(ctypes.byref(stream), 0) == 0
        popped = ctypes.c_void_p()
        assert cu.cuCtxPopCurrent_v2(ctypes.byref(popped)) == 0   # back to the primary context
        W, H, pose, cam, depth, state = inputs(5, 64, 48)
        N = W * H
        bufs = [torch.zeros(N, dtype=torch.float32, device="cuda") for _ in range(10)]
        ptrs = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in bufs[2:6]])
        ptrs2 = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in bufs[6:10]])
        st = pm_lib.pm_stage_depth_fuse_noalloc(W, H, fptr(pose), fptr(cam), vp(bufs[0]), ptrs, ptrs2,
                                                ctypes.c_void_p(0), stream)
        assert st == 1   # PM_ERR_INVALID_ARGUMENT
        assert cu.cuCtxPushCurrent_v2(ctx) == 0
        assert cu.cuStreamDestroy_v2(stream) == 0
        assert cu.cuCtxPopCurrent_v2(ctypes.byref(popped)) == 0
    finally:
        assert cu.cuCtxDestroy_v2(ctx) == 0


def test_noalloc_rejects_images_beyond_its_array(pm_lib):
    W, H = 1024, 1024   # 2^20 pixels, above the 2^19 limit; rejected before any GPU work
    pose = np.eye(3, dtype=np.float32).reshape(-1).tolist() + [0.0, 0.0, 0.0]
    pose = np.array(pose, np.float32)
    cam = np.array([500, 500, 512, 512], np.float32)
    ptrs = (ctypes.c_void_p * 4)(*([1] * 4))
    st = pm_lib.pm_stage_depth_fuse_noalloc(W, H, fptr(pose), fptr(cam), ctypes.c_void_p(1), ptrs, ptrs,
                                            ctypes.c_void_p(0), None)
    assert st == 1   # PM_ERR_INVALID_ARGUMENT
