"""CPU restatement of the reference driver's keyframe schedule -- TEST INFRASTRUCTURE, NOT
PRODUCT CODE.  Only tests/ import this module, as the checker of the pm_sequence driver
(probabilistic_mapping_b200/cli/pm_sequence.cpp).

evaluate.cc keeps images and poses in two lists that grow at the front (GrabImage / GrabPose,
evaluate.cc:87-116).  processImg (evaluate.cc:137-239):
  * returns while the image list holds no more than lastSize entries (lastSize starts at
    aggNum * interval, evaluate.cc:348);
  * returns while the newest pose is older than the newest image (:169-171);
  * searches the pose with the newest image's timestamp from the newest pose on (:183-205) and
    returns with a warning when there is none;
  * takes the images interval, 2 interval, ... places older than the newest, and the poses the same
    number of places older than the matched one (:210-231);
  * increments lastSize and drops the oldest image and pose (:232-235).
Offline replay: the poses up to an image's time arrive before it; after each arrival
processImg runs until it returns without a keyframe.  Where the reference would step past the
end of the pose list (undefined behaviour) the restatement stops with a warning.
"""
from __future__ import annotations

from collections import deque


def stamp_ns(text: str) -> int:
    ip, _, fp = text.partition(".")
    return int(ip) * 10 ** 9 + int((fp + "0" * 9)[:9])


def schedule(images, poses, agg=3, interval=6):
    """images: [(stamp_text, file)], poses: [(stamp_text, ...)].  Returns (keyframes, warnings),
    each keyframe (ref_index, ref_pose_index, [(src_index, src_pose_index)])."""
    fo = sorted(range(len(images)), key=lambda i: stamp_ns(images[i][0]))
    po = sorted(range(len(poses)), key=lambda i: stamp_ns(poses[i][0]))
    it = lambda i: stamp_ns(images[i][0])
    pt = lambda i: stamp_ns(poses[i][0])
    img, pos = deque(), deque()
    last = agg * interval
    warnings = 0
    out = []

    def process():
        nonlocal last, warnings
        if len(img) <= last:
            return None
        if not pos or pt(pos[0]) < it(img[0]):
            return None
        ip = next((k for k, p in enumerate(pos) if pt(p) == it(img[0])), None)
        if ip is None:
            warnings += 1
            return None
        if ip + agg * interval >= len(pos):
            warnings += 1
            return None
        kf = (img[0], pos[ip], [(img[i * interval], pos[ip + i * interval]) for i in range(1, agg + 1)])
        last += 1
        img.pop()
        pos.pop()
        return kf

    pi = 0
    for f in fo:
        while pi < len(po) and pt(po[pi]) <= it(f):
            pos.appendleft(po[pi])
            pi += 1
        img.appendleft(f)
        while (k := process()) is not None:
            out.append(k)
    while pi < len(po):
        pos.appendleft(po[pi])
        pi += 1
    while (k := process()) is not None:
        out.append(k)
    return out, warnings
