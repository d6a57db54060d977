"""The keyframe schedule of the headless driver (pm_sequence --dry-run, no GPU) against the
restatement of evaluate.cc:137-239 in oracle/sequence.py, on streams that exercise every branch:
aligned images and poses, missing poses, poses at a higher rate, late poses, unsorted lists, and
restamping with --associate."""
import os

import numpy as np
import pytest

from oracle import sequence as oseq


@pytest.fixture(scope="module")
def cli(pm_lib):
    from probabilistic_mapping_b200 import build
    return build.build_cli()


def write_lists(tmp, images, poses):
    il, pl = os.path.join(tmp, "rgb.txt"), os.path.join(tmp, "poses.txt")
    with open(il, "w") as f:
        f.write("# timestamp filename\n")
        for st, name in images:
            f.write(f"{st} {name}\n")
    with open(pl, "w") as f:
        for st, *_ in poses:
            f.write(f"{st} 0.1 0.2 0.3 0 0 0 1\n")
    return il, pl


def dry(tmp, images, poses, **opts):
    from probabilistic_mapping_b200 import sequence
    il, pl = write_lists(tmp, images, poses)
    out = sequence.run(il, pl, str(tmp), dry_run=True, **opts)
    return out[:-1], out[-1]


def expected(images, poses, agg=3, interval=6):
    kfs, warn = oseq.schedule(images, poses, agg, interval)
    rows = [{"ref": images[r][0], "ref_file": images[r][1], "ref_pose": poses[rp][0],
             "sources": [[images[s][0], poses[sp][0]] for s, sp in src]} for r, rp, src in kfs]
    return rows, warn


def stamps(n, t0=100.0, dt=1 / 30):
    return [f"{t0 + k * dt:.6f}" for k in range(n)]


def check(tmp, images, poses, **kw):
    rows, summary = dry(tmp, images, poses, **{k: v for k, v in kw.items() if k in ("agg", "interval")})
    want, warn = expected(images, poses, kw.get("agg", 3), kw.get("interval", 6))
    assert rows == want
    assert summary == {"keyframes": len(want), "warnings": warn}
    return rows, warn


def test_aligned_stream(cli, tmp_path):
    st = stamps(60)
    images = [(s, f"rgb/{s}.png") for s in st]
    rows, warn = check(str(tmp_path), images, [(s,) for s in st])
    # the first keyframe once 19 frames are in, then every second frame; sources 6, 12, 18 back
    assert [r["ref"] for r in rows] == st[18::2]
    assert rows[0]["sources"] == [[st[12], st[12]], [st[6], st[6]], [st[0], st[0]]]
    assert warn == 0


def test_custom_agg_and_interval(cli, tmp_path):
    st = stamps(40)
    check(str(tmp_path), [(s, f"{s}.pgm") for s in st], [(s,) for s in st], agg=2, interval=4)


def test_missing_poses(cli, tmp_path):
    st = stamps(70)
    rng = np.random.default_rng(0)
    keep = [s for s in st if rng.random() > 0.15]
    _, warn = check(str(tmp_path), [(s, f"{s}.png") for s in st], [(s,) for s in keep])
    assert warn > 0


def test_poses_at_three_times_the_image_rate(cli, tmp_path):
    st = stamps(50)
    fine = stamps(150, dt=1 / 90)          # includes every image stamp
    assert set(st) <= set(fine)
    rows, _ = check(str(tmp_path), [(s, f"{s}.png") for s in st], [(s,) for s in fine])
    # the reference steps through the pose list by position, so the sources' poses are not theirs
    assert rows and rows[0]["sources"][0][0] != rows[0]["sources"][0][1]


def test_late_and_unsorted_lists(cli, tmp_path):
    st = stamps(45)
    images = [(s, f"{s}.png") for s in st]
    poses = [(s,) for s in st[:30]]        # the pose stream stops early
    rng = np.random.default_rng(1)
    check(str(tmp_path), [images[i] for i in rng.permutation(len(images))], poses)


def test_associate_restamps_nearest_pose(cli, tmp_path):
    from probabilistic_mapping_b200 import sequence
    st = stamps(40)
    jitter = [f"{float(s) + 0.004:.6f}" for s in st]
    images = [(s, f"{s}.png") for s in st]
    il, pl = write_lists(str(tmp_path), images, [(s,) for s in jitter])
    exact = sequence.run(il, pl, str(tmp_path), dry_run=True)
    assert exact[-1]["keyframes"] == 0     # exact matching finds no pose
    assoc = sequence.run(il, pl, str(tmp_path), dry_run=True, associate=0.01)
    want, _ = expected(images, [(s,) for s in st])
    assert assoc[:-1] == want
