"""Build recipe for libpm_stereo.so (sm_100a).

Compiles every .cu under csrc/ with nvcc for sm_100a (and the host-only .cpp files there with
g++) and links one shared library next to this file.  -fmad=false: FP32 expressions are written with explicit fused/unfused
intrinsics, so the compiler must not contract multiply-adds on its own (the CPU oracle replays
the same operation order).

The same sources also build libpm_stereo_checked.so: -DPM_BOUNDS_CHECK turns on the element-index
tests of the kernels' global accesses (a failing access is skipped and recorded, read back with
pm_debug_bounds), and relocatable device code lets all kernels share one record.  It is a test
build; the product library is libpm_stereo.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpm_stereo.so")
LIB_CHECKED = os.path.join(HERE, "libpm_stereo_checked.so")
BUILD_CHECKED = os.path.join(HERE, "_build_checked")
CHECKED_FLAGS = ["-DPM_BOUNDS_CHECK", "-rdc=true"]
CLI_SRC = os.path.join(HERE, "cli", "pm_sequence.cpp")
CLI = os.path.join(HERE, "pm_sequence")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
                     "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libpm_stereo.so")
    return path


CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _host_sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps_mtime() -> float:
    files = _sources() + _host_sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h")) + [os.path.abspath(__file__)]
    return max(os.path.getmtime(f) for f in files)


def cuda_home() -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))


def build_cli(force: bool = False) -> str:
    """The headless sequence driver: cli/pm_sequence.cpp linked against libpm_stereo.so (found
    next to the binary through its rpath) and the static CUDA runtime."""
    newest = max(os.path.getmtime(CLI_SRC), os.path.getmtime(LIB),
                 max(os.path.getmtime(f) for f in glob.glob(os.path.join(ROOT, "include", "*.h"))))
    if not force and os.path.exists(CLI) and os.path.getmtime(CLI) >= newest:
        return CLI
    cuda = cuda_home()
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(cuda, "include"),
           CLI_SRC, "-o", CLI + ".tmp", "-L", HERE, "-lpm_stereo", "-Wl,-rpath,$ORIGIN",
           "-L", os.path.join(cuda, "lib64"), "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building pm_sequence failed:\n{r.stdout}\n{r.stderr}")
    os.replace(CLI + ".tmp", CLI)
    return CLI


def _compile(src: str, extra: list[str], outdir: str = BUILD) -> str:
    obj = os.path.join(outdir, os.path.basename(src) + ".o")
    cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def _compile_host(src: str) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cxx = shutil.which("g++") or "g++"
    r = subprocess.run([cxx] + CXX_FLAGS + ["-c", src, "-o", obj], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def _link(objs: list[str], lib: str, extra: list[str]) -> None:
    tmp = lib + ".tmp"
    cmd = [nvcc()] + ARCH + extra + ["-shared", "-o", tmp] + objs + ["-lcuda", "-lz"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)


def build(force: bool = False, verbose_ptxas: bool = False, checked: bool = True) -> str:
    """Compile csrc/*.cu for sm_100a into libpm_stereo.so and, with `checked`, the bounds-checked
    libpm_stereo_checked.so (each skipped when up to date)."""
    deps = _deps_mtime()
    need = force or not os.path.exists(LIB) or os.path.getmtime(LIB) < deps
    need_checked = checked and (force or not os.path.exists(LIB_CHECKED) or os.path.getmtime(LIB_CHECKED) < deps)
    if not need and not need_checked:
        build_cli()
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(BUILD_CHECKED, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        jobs = [ex.submit(_compile, s, extra) for s in _sources()] if need else []
        cjobs = [ex.submit(_compile, s, CHECKED_FLAGS, BUILD_CHECKED) for s in _sources()] if need_checked else []
        host = list(ex.map(_compile_host, _host_sources()))
        objs = [j.result() for j in jobs]
        cobjs = [j.result() for j in cjobs]
    if need:
        _link(objs + host, LIB, [])
    if need_checked:
        _link(cobjs + host, LIB_CHECKED, ["-rdc=true"])
    build_cli(force=need)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
    print(LIB)
