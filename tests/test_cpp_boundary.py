"""The C++ StereoMapper header compiles and links against libpm_stereo.so like a host
program of the reference would, and reports errors as pm::Error."""
import os
import subprocess

import pytest

from conftest import ROOT


def build_smoke(tmp_path):
    exe = tmp_path / "mapper_smoke"
    lib_dir = os.path.join(ROOT, "probabilistic_mapping_b200")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "mapper_smoke.cpp"), "-L", lib_dir, "-lpm_stereo",
           f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True)
    return exe


def test_cpp_header_builds_and_reports_errors(pm_lib, tmp_path):
    exe = build_smoke(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_header_maps_a_frame(pm_lib, tmp_path):
    exe = build_smoke(tmp_path)
    r = subprocess.run([str(exe), "gpu"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
