"""Build recipe for oracle/_ref/ -- TEST INFRASTRUCTURE.

Compiles the reference's motion_stereo/*.cu (HKUST-Aerial-Robotics/probabilistic_mapping,
read from /root/reference where they lie; nothing is copied) with oracle/ref_shim.h
force-included and oracle/ref_unity.cu as the translation unit, once per test shape, into
oracle/_ref/libref_<W>x<H>x<D>.so.  The reference's default nvcc settings are kept (FMA
contraction on), so the library behaves like the reference built for sm_100a.  Needs the
reference sources, so it runs only where they are present; the built libraries travel with
the repository snapshot to GPU hosts.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = "/root/reference/motion_stereo"
OUT = os.path.join(HERE, "_ref")
SHAPES = [(40, 32, 32), (640, 480, 64)]


def lib_path(W: int, H: int, D: int) -> str:
    return os.path.join(OUT, f"libref_{W}x{H}x{D}.so")


def build(shapes=SHAPES, force: bool = False) -> list[str]:
    if not os.path.isdir(REF_SRC):
        raise RuntimeError(f"reference sources not found at {REF_SRC}")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    os.makedirs(OUT, exist_ok=True)
    deps = [os.path.join(HERE, "ref_shim.h"), os.path.join(HERE, "ref_unity.cu")]
    built = []
    for W, H, D in shapes:
        out = lib_path(W, H, D)
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
            built.append(out)
            continue
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++14", "-Xcompiler", "-fPIC",
               "-shared", "-w", "-I", REF_SRC, "-include", os.path.join(HERE, "ref_shim.h"),
               f"-DPM_REF_W={W}", f"-DPM_REF_H={H}", f"-DPM_REF_D={D}", os.path.join(HERE, "ref_unity.cu"),
               "-o", out]
        subprocess.run(cmd, check=True)
        built.append(out)
    return built


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv):
        print(p)
