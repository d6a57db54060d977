"""The headless sequence driver (pm_sequence, in place of evaluate.cc) end to end on a synthetic
TUM-style stream written to disk: its depth files are compared bit-for-bit with the same keyframe
schedule (oracle/sequence.py) driven through the Python StereoMapper, with the pyramid and
colour steps checked against oracle/imgproc.py."""
import os

import numpy as np
import pytest

from oracle import imgproc as oip
from oracle import sequence as oseq
from probabilistic_mapping_b200 import _lib, scene, sequence
from probabilistic_mapping_b200.mapper import StereoMapper

pytestmark = pytest.mark.gpu

W, H, F, N = 160, 120, 130.0, 27


@pytest.fixture(scope="module")
def stream(tmp_path_factory, pm_lib):
    from probabilistic_mapping_b200 import build
    build.build_cli()
    root = str(tmp_path_factory.mktemp("seq"))
    imgs, R, T, K = scene.make_stream(W, H, F, N, seed=5)
    il, pl = sequence.write_tum(root, imgs, R, T)
    images = [tuple(l.split()) for l in open(il) if not l.startswith("#")]
    poses = [l.split() for l in open(pl) if not l.startswith("#")]
    return dict(root=root, il=il, pl=pl, imgs=imgs, images=images, poses=poses)


def python_run(st, case, downsample=0):
    """evaluate.cc's keyframe loop through the Python StereoMapper, on the oracle's schedule."""
    kfs, _ = oseq.schedule(st["images"], [(p[0],) for p in st["poses"]])
    fx, fy, cx, cy = F, F, W / 2.0, H / 2.0
    for _ in range(downsample):
        fx, fy, cx, cy = fx / 2, fy / 2, (cx + 0.5) / 2.0 - 0.5, (cy + 0.5) / 2.0 - 0.5
    K = np.array([[fx, 0, cx], [0, fy, cy], [0, 0, 1.0]])

    def frame(i):
        img = st["imgs"][i]
        for _ in range(downsample):
            img = oip.pyr_down(img)
        return img

    def pose(i):
        p = [float(v) for v in st["poses"][i][1:]]
        return sequence.quat_to_rot(p[3], p[4], p[5], p[6]), np.array(p[:3])

    w, h = W >> downsample, H >> downsample
    m = StereoMapper(w, h, 64, fusion_variant=_lib.PM_FUSION_CPU_PATH, max_sources=3)
    m.initIntrinsic(K, 0.02 * fx, np.float32(1.0 / (0.15 * 160.0)))
    out = {}
    for ref, rp, src in kfs:
        Rl, Tl = pose(rp)
        m.initReference(frame(ref))
        for s, sp in src:
            Rr, Tr = pose(sp)
            m.update(frame(s), Rl, Tl, Rr, Tr)
        if case >= 3:
            d, _ = m.outputFusion(Rl, Tl, fx, fy, cx, cy, want_variance=False)
        else:
            d = m.outputCase(case)
        for _ in range(downsample):
            d = oip.depth_up2(d)
        out[st["images"][ref][0]] = d
    m.close()
    return out


def cli_run(st, tmp, case, downsample=0, fmt="pfm", color=True):
    os.makedirs(tmp, exist_ok=True)
    res = sequence.run(st["il"], st["pl"], tmp, root=st["root"], case=case, downsample=downsample,
                       fx=repr(F), fy=repr(F), cx=repr(W / 2.0), cy=repr(H / 2.0), format=fmt, color=color)
    return res[-1]


def read_ppm(path):
    data = open(path, "rb").read()
    parts = data.split(b"\n", 3)
    w, h = (int(v) for v in parts[1].split())
    rgb = np.frombuffer(parts[3], np.uint8, count=w * h * 3).reshape(h, w, 3)
    return rgb[..., ::-1]


@pytest.mark.parametrize("case,downsample", [(3, 0), (3, 1), (0, 0), (1, 1)])
def test_driver_matches_python_loop(stream, tmp_path, case, downsample):
    summary = cli_run(stream, str(tmp_path), case, downsample)
    want = python_run(stream, case, downsample)
    assert summary["keyframes"] == len(want) == 5 and summary["warnings"] == 0
    assert (summary["width"], summary["height"]) == (W, H)
    nonzero = 0
    for stamp, d in want.items():
        got = sequence.read_pfm(os.path.join(str(tmp_path), f"depth_{stamp}.pfm"))
        assert got.shape == (H, W)
        assert (got.view(np.uint32) == d.view(np.uint32)).all(), stamp
        nonzero += int(((d > 0) & (d < 100)).sum())
        level, bgr = oip.colorize(oip.range_mask(d, 0.2, 20.0))
        np.testing.assert_array_equal(read_ppm(os.path.join(str(tmp_path), f"color_{stamp}.ppm")), bgr)
    assert nonzero > 0


def oracle_run(st, case, downsample=0):
    """The same keyframe loop through the CPU oracle (FP32 instantiation, the CPU fusion
    variant for CASE >= 3, the CASE argmin for CASE 0 / 1), with the reference's parameters
    (parameters.cpp:12-18, 64 planes, 4 paths, DEP_SAMPLE of evaluate.cc:345) and the oracle's
    pyrDown / up-sampling: the driver's files are checked against it, not against itself."""
    import oracle
    kfs, _ = oseq.schedule(st["images"], [(p[0],) for p in st["poses"]])
    fx, fy, cx, cy = F, F, W / 2.0, H / 2.0
    for _ in range(downsample):
        fx, fy, cx, cy = fx / 2, fy / 2, (cx + 0.5) / 2.0 - 0.5, (cy + 0.5) / 2.0 - 0.5
    K = np.array([[fx, 0, cx], [0, fy, cy], [0, 0, 1.0]])
    w, h = W >> downsample, H >> downsample
    drho = float(np.float32(1.0 / (0.15 * 160.0)))
    o = oracle.Mapper(oracle.Params(W=w, H=h, D=64, drho=drho), K, prec="f32", fusion="cpu")

    def frame(i):
        img = st["imgs"][i]
        for _ in range(downsample):
            img = oip.pyr_down(img)
        return img

    def pose(i):
        p = [float(v) for v in st["poses"][i][1:]]
        return sequence.quat_to_rot(p[3], p[4], p[5], p[6]), np.array(p[:3])

    out = {}
    for ref, rp, src in kfs:
        Rl, Tl = pose(rp)
        o.init_reference(frame(ref))
        for s, sp in src:
            Rr, Tr = pose(sp)
            o.update(frame(s), Rl, Tl, Rr, Tr)
        if case >= 3:
            d = o.output_fusion(Rl, Tl, np.float32(fx), np.float32(fy), np.float32(cx), np.float32(cy))["fused"]
        else:
            stg = o.stages()
            vol = stg["cost"] if case == 0 else stg["sgm"]
            d, _ = oip.case_argmin(vol.reshape(h, w, 64), 0.0, drho)
        d = np.asarray(d, np.float32)
        for _ in range(downsample):
            d = oip.depth_up2(d)
        out[st["images"][ref][0]] = d
    return out


@pytest.mark.parametrize("case,downsample", [(3, 0), (3, 1), (0, 0), (1, 1)])
def test_driver_matches_oracle(stream, tmp_path, case, downsample):
    """The driver's depth files against the oracle run over the same schedule: CASE 0 / 1
    bit-exact; the fused depth of CASE 3 with the same zero / non-zero pattern and within 1e-4
    relative (CUDA's expf in the update against the host's)."""
    summary = cli_run(stream, str(tmp_path), case, downsample, color=False)
    want = oracle_run(stream, case, downsample)
    assert summary["keyframes"] == len(want) == 5
    fused = 0
    for stamp, d in want.items():
        got = sequence.read_pfm(os.path.join(str(tmp_path), f"depth_{stamp}.pfm"))
        if case < 3:
            assert (got.view(np.uint32) == d.view(np.uint32)).all(), stamp
        else:
            assert ((got == 0) == (d == 0)).mean() >= 0.999, stamp
            both = (got != 0) & (d != 0)
            np.testing.assert_allclose(got[both], d[both], rtol=1e-4, err_msg=stamp)
            fused += int(both.sum())
    assert case < 3 or fused > 0


def test_driver_fp16_texture(stream, tmp_path):
    """The FP16 form with the texture sampler through the driver: same files as the Python loop
    with the same configuration."""
    os.makedirs(str(tmp_path), exist_ok=True)
    sequence.run(stream["il"], stream["pl"], str(tmp_path), root=stream["root"], case=3, fx=repr(F), fy=repr(F),
                 cx=repr(W / 2.0), cy=repr(H / 2.0), precision="fp16", sampler="texture_f32")
    kfs, _ = oseq.schedule(stream["images"], [(p[0],) for p in stream["poses"]])
    K = np.array([[F, 0, W / 2.0], [0, F, H / 2.0], [0, 0, 1.0]])
    m = StereoMapper(W, H, 64, fusion_variant=_lib.PM_FUSION_CPU_PATH, max_sources=3,
                     precision=_lib.PM_PREC_FP16, sampler=_lib.PM_SAMPLER_TEXTURE_F32)
    m.initIntrinsic(K, 0.02 * F, np.float32(1.0 / (0.15 * 160.0)))

    def pose(i):
        p = [float(v) for v in stream["poses"][i][1:]]
        return sequence.quat_to_rot(p[3], p[4], p[5], p[6]), np.array(p[:3])

    for ref, rp, src in kfs:
        Rl, Tl = pose(rp)
        m.initReference(stream["imgs"][ref])
        for s, sp in src:
            Rr, Tr = pose(sp)
            m.update(stream["imgs"][s], Rl, Tl, Rr, Tr)
        d, _ = m.outputFusion(Rl, Tl, F, F, W / 2.0, H / 2.0, want_variance=False)
        got = sequence.read_pfm(os.path.join(str(tmp_path), f"depth_{stream['images'][ref][0]}.pfm"))
        assert (got.view(np.uint32) == d.view(np.uint32)).all()
    m.close()


def test_driver_npy_output(stream, tmp_path):
    cli_run(stream, str(tmp_path), 2, 0, fmt="npy", color=False)
    want = python_run(stream, 2)
    for stamp, d in want.items():
        np.testing.assert_array_equal(np.load(os.path.join(str(tmp_path), f"depth_{stamp}.npy")), d)


def test_driver_time_per_keyframe_640x480(tmp_path_factory):
    """Measurement: the driver's mean time per keyframe (initReference, three updates, the CPU
    fusion variant, copy-out; the interval evaluate.cc:244-269 times) at 640x480 with the
    reference's 64 planes and 4 paths, FP32 and FP16 with the texture sampler.  With
    PM_REPORT_DIR set the numbers go to $PM_REPORT_DIR/driver_640x480.json."""
    import json
    root = str(tmp_path_factory.mktemp("seq640"))
    imgs, R, T, _ = scene.make_stream(640, 480, 520.0, 25, seed=6, step=0.02)
    il, pl = sequence.write_tum(root, imgs, R, T)
    report = {}
    for name, opts in (("fp32", {}), ("fp16_texture_f32", dict(precision="fp16", sampler="texture_f32"))):
        out = os.path.join(root, name)
        os.makedirs(out)
        res = sequence.run(il, pl, out, root=root, case=3, fx="520.0", fy="520.0", cx="320.0", cy="240.0", **opts)
        report[name] = res[-1]
    print(json.dumps(report))
    rep = os.environ.get("PM_REPORT_DIR")
    if rep:
        os.makedirs(rep, exist_ok=True)
        with open(os.path.join(rep, "driver_640x480.json"), "w") as f:
            json.dump(report, f, indent=1)
    assert all(r["keyframes"] == 4 and r["mean_ms_per_keyframe"] > 0 for r in report.values())
