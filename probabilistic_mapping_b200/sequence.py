"""Sequences on disk for the headless driver (probabilistic_mapping_b200/pm_sequence, the
counterpart of the reference's ROS node evaluate.cc).

* ``write_tum``: an image list, a pose list (camera-to-world, "timestamp tx ty tz qx qy qz qw")
  and 8-bit PNG or PGM frames -- the layout of the TUM RGB-D / ICL-NUIM sequences the reference
  was run on (evaluate.cc:30-40).
* ``rot_to_quat`` / ``quat_to_rot``: the quaternion convention of those files;
  ``quat_to_rot`` is Eigen's toRotationMatrix formula (evaluate.cc:190-195), as the driver uses.
* ``read_pfm``: reads the driver's depth output.
* ``run``: runs the driver binary.
"""
from __future__ import annotations

import json
import os
import struct
import subprocess
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CLI = os.path.join(HERE, "pm_sequence")


def rot_to_quat(R) -> tuple[float, float, float, float]:
    """Unit quaternion (x, y, z, w) of a rotation matrix (Shepperd's method)."""
    R = np.asarray(R, np.float64)
    tr = np.trace(R)
    if tr > 0:
        s = 2.0 * np.sqrt(tr + 1.0)
        w, x, y, z = 0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s
    else:
        i = int(np.argmax(np.diag(R)))
        j, k = (i + 1) % 3, (i + 2) % 3
        s = 2.0 * np.sqrt(1.0 + R[i, i] - R[j, j] - R[k, k])
        q = np.zeros(4)
        q[i] = 0.25 * s
        q[j] = (R[j, i] + R[i, j]) / s
        q[k] = (R[k, i] + R[i, k]) / s
        w = (R[k, j] - R[j, k]) / s
        x, y, z = q[0], q[1], q[2]
    return float(x), float(y), float(z), float(w)


def quat_to_rot(x, y, z, w) -> np.ndarray:
    """Eigen's Quaternion::toRotationMatrix (no normalisation), the driver's conversion."""
    tx, ty, tz = 2 * x, 2 * y, 2 * z
    twx, twy, twz = tx * w, ty * w, tz * w
    txx, txy, txz = tx * x, ty * x, tz * x
    tyy, tyz, tzz = ty * y, tz * y, tz * z
    return np.array([[1 - (tyy + tzz), txy - twz, txz + twy],
                     [txy + twz, 1 - (txx + tzz), tyz - twx],
                     [txz - twy, tyz + twx, 1 - (txx + tyy)]])


def write_png_grey(path: str, img: np.ndarray) -> None:
    """8-bit greyscale PNG (filter type 0 on every row, zlib-compressed)."""
    img = np.ascontiguousarray(img, np.uint8)
    H, W = img.shape

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xffffffff)

    raw = b"".join(b"\x00" + img[y].tobytes() for y in range(H))
    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, 8, 0, 0, 0, 0)) +
                chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


def write_pgm(path: str, img: np.ndarray) -> None:
    img = np.ascontiguousarray(img, np.uint8)
    with open(path, "wb") as f:
        f.write(b"P5\n%d %d\n255\n" % (img.shape[1], img.shape[0]) + img.tobytes())


def write_tum(root: str, images, R, T, t0: float = 1000.0, dt: float = 1.0 / 30.0, fmt: str = "png",
              pose_stamps=None) -> tuple[str, str]:
    """Writes frames and the two lists under root; returns (image list, pose list) paths.
    Timestamps are t0 + k dt with six decimals; pose_stamps (optional) overrides the pose
    timestamps (strings)."""
    os.makedirs(os.path.join(root, "rgb"), exist_ok=True)
    il, pl = os.path.join(root, "rgb.txt"), os.path.join(root, "groundtruth.txt")
    with open(il, "w") as fi, open(pl, "w") as fp:
        fi.write("# timestamp filename\n")
        fp.write("# timestamp tx ty tz qx qy qz qw\n")
        for k, img in enumerate(images):
            st = f"{t0 + k * dt:.6f}"
            name = f"rgb/{st}.{fmt}"
            (write_png_grey if fmt == "png" else write_pgm)(os.path.join(root, name), img)
            fi.write(f"{st} {name}\n")
        for k in range(len(R)):
            st = pose_stamps[k] if pose_stamps is not None else f"{t0 + k * dt:.6f}"
            vals = [float(v) for v in T[k]] + list(rot_to_quat(R[k]))
            fp.write(st + "".join(f" {v!r}" for v in vals) + "\n")
    return il, pl


def read_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        data = f.read()
    parts = data.split(b"\n", 3)
    if parts[0] != b"Pf":
        raise ValueError("not a greyscale PFM")
    W, H = (int(v) for v in parts[1].split())
    scale = float(parts[2])
    arr = np.frombuffer(parts[3], dtype="<f4" if scale < 0 else ">f4", count=W * H).reshape(H, W)
    return arr[::-1].astype(np.float32)


def run(images: str, poses: str, out: str, root: str | None = None, dry_run: bool = False, **opts):
    """Runs pm_sequence; opts become --key value flags (True for bare flags).  Returns the JSON
    objects it printed."""
    if not os.path.exists(CLI):
        raise RuntimeError(f"{CLI} is missing: run probabilistic_mapping_b200/build.py")
    cmd = [CLI, "--images", images, "--poses", poses, "--out", out]
    if root:
        cmd += ["--root", root]
    if dry_run:
        cmd.append("--dry-run")
    for k, v in opts.items():
        flag = "--" + k.replace("_", "-")
        if v is True:
            cmd.append(flag)
        elif v is not False and v is not None:
            cmd += [flag, str(v)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"pm_sequence failed ({r.returncode}): {r.stderr.strip()}")
    return [json.loads(line) for line in r.stdout.splitlines() if line.strip()]
