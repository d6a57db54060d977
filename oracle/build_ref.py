"""Build recipe for oracle/_ref/ -- TEST INFRASTRUCTURE.

Compiles the reference's motion_stereo/*.cu (HKUST-Aerial-Robotics/probabilistic_mapping,
read where they lie -- $PM_REFERENCE_ROOT/motion_stereo, by default under /root/reference --
nothing is copied) with oracle/ref_shim.h
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
REF_ROOT = os.environ.get("PM_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "motion_stereo")
OUT = os.path.join(HERE, "_ref")
SHAPES = [(40, 32, 32), (640, 480, 64)]


def available() -> bool:
    """True where the reference sources are present (the container that builds; not GPU hosts)."""
    return os.path.isdir(REF_SRC)


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


CPU_SHAPES = [(80, 60, 32)]


def cpu_lib_path(W: int, H: int, D: int) -> str:
    return os.path.join(OUT, f"libref_cpu_{W}x{H}x{D}.so")


def build_cpu(shapes=CPU_SHAPES, force: bool = False) -> list[str]:
    """The reference's stereo_mapper.cpp (its CPU fusion variant and CASE outputs) compiled on the
    host, unmodified, through oracle/ref_cpu_unity.cpp against the stand-in headers of
    oracle/ref_stubs/.  Multiply-adds are not contracted (-ffp-contract=off): the library
    evaluates the source's expressions as written.  (The reference's own build uses
    -march=native, where g++ may fuse multiply-adds on hosts with FMA units.)"""
    if not available():
        raise RuntimeError(f"reference sources not found at {REF_SRC}")
    cxx = shutil.which("g++") or "g++"
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(
        shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"))), "include")
    os.makedirs(OUT, exist_ok=True)
    deps = [os.path.join(HERE, "ref_cpu_unity.cpp"), os.path.join(HERE, "ref_params.h")]
    for root, _, files in os.walk(os.path.join(HERE, "ref_stubs")):
        deps += [os.path.join(root, f) for f in files]
    built = []
    for W, H, D in shapes:
        out = cpu_lib_path(W, H, D)
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
            built.append(out)
            continue
        cmd = [cxx, "-O2", "-std=c++14", "-fPIC", "-shared", "-w", "-ffp-contract=off",
               "-I", os.path.join(HERE, "ref_stubs"), "-I", REF_SRC, "-I", cuda_inc,
               "-include", os.path.join(HERE, "ref_params.h"),
               f"-DPM_REF_W={W}", f"-DPM_REF_H={H}", f"-DPM_REF_D={D}", os.path.join(HERE, "ref_cpu_unity.cpp"),
               "-o", out]
        subprocess.run(cmd, check=True)
        built.append(out)
    return built


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv) + build_cpu(force="--force" in sys.argv):
        print(p)
