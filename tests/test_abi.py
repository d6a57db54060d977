"""The C-ABI library loads, exports every entry point declared in include/pm_stereo.h, and
rejects bad arguments with status codes (no GPU needed for any of this)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pm_stereo.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"PM_API\s+[\w\s\*]+?\b(pm_\w+)\s*\(", text)))


def test_header_declarations_are_exported(pm_lib):
    names = declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(pm_lib, n), f"{n} is declared in pm_stereo.h but not exported"
    from probabilistic_mapping_b200 import _lib
    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures and header disagree"


def test_build_targets_sm100a_only():
    from probabilistic_mapping_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-fmad=false" in build.NVCC_FLAGS


def test_config_defaults_are_the_reference_parameters(pm_lib):
    from probabilistic_mapping_b200 import _lib
    c = _lib.default_config(640, 480, 64)
    assert (c.p1, c.p2, c.tau_so, c.q1, c.q2) == (8.0, 24.0, 4.0, 2.0, 3.0)      # parameters.cpp:12-16
    assert abs(c.var_scale - 1.02) < 1e-7                                           # parameters.cpp:18
    assert abs(c.rho_step - 1 / (0.15 * 160)) < 1e-8                                # evaluate.cc:345
    assert c.rho0 == 0.0 and c.num_paths == 4 and c.cost_mode == _lib.PM_COST_REFERENCE
    assert c.intensity_scale == 1.0 and c.tree_compat == 1


@pytest.mark.parametrize("field,value", [("num_planes", 48), ("num_planes", 512), ("num_paths", 6),
                                         ("width", 2), ("cost_mode", 7), ("max_sources", 0),
                                         ("rho_step", 0.0), ("precision", 9)])
def test_create_rejects_bad_config(pm_lib, field, value):
    from probabilistic_mapping_b200 import _lib
    c = _lib.default_config(64, 48, 64)
    setattr(c, field, value)
    h = ctypes.c_void_p()
    assert pm_lib.pm_create(ctypes.byref(c), ctypes.byref(h)) == _lib.PM_ERR_INVALID_ARGUMENT
    assert not h.value


def test_fp16_texels_belong_to_the_fp16_form(pm_lib):
    """The FP32 form takes the exact sampler or the texture unit on FP32 texels; FP16 texels (and
    unknown samplers) are rejected before any device work."""
    from probabilistic_mapping_b200 import _lib
    for precision, sampler in ((_lib.PM_PREC_FP32, _lib.PM_SAMPLER_TEXTURE), (_lib.PM_PREC_FP32, 5),
                               (_lib.PM_PREC_FP16, 3)):
        c = _lib.default_config(64, 48, 64)
        c.precision, c.sampler = precision, sampler
        h = ctypes.c_void_p()
        assert pm_lib.pm_create(ctypes.byref(c), ctypes.byref(h)) == _lib.PM_ERR_INVALID_ARGUMENT
        assert not h.value


def test_fp16_needs_even_planes_per_lane(pm_lib):
    from probabilistic_mapping_b200 import _lib
    c = _lib.default_config(64, 48, 96)
    c.precision = _lib.PM_PREC_FP16
    h = ctypes.c_void_p()
    assert pm_lib.pm_create(ctypes.byref(c), ctypes.byref(h)) == _lib.PM_ERR_INVALID_ARGUMENT


def test_stage_calls_validate_arguments(pm_lib):
    from probabilistic_mapping_b200 import _lib
    c = _lib.default_config(64, 48, 64)
    null = ctypes.c_void_p(0)
    assert pm_lib.pm_stage_sgm(ctypes.byref(c), null, null, null, null, null) == _lib.PM_ERR_INVALID_ARGUMENT
    assert pm_lib.pm_stage_filter(ctypes.byref(c), null, null, 0, null, null) == _lib.PM_ERR_INVALID_ARGUMENT
    assert pm_lib.pm_stage_convert(64, 48, null, null, 1, 4, null) == _lib.PM_ERR_INVALID_ARGUMENT
    assert pm_lib.pm_stage_to_float(0, 48, null, 64, null, 1.0, null) == _lib.PM_ERR_INVALID_ARGUMENT
    f = (ctypes.c_float * 12)()
    assert pm_lib.pm_stage_calc_cost(ctypes.byref(c), null, null, 1, f, null, null, null, null) == \
        _lib.PM_ERR_INVALID_ARGUMENT
    assert pm_lib.pm_status_string(_lib.PM_ERR_BAD_STATE) == b"bad state"


def test_create_without_device_fails_cleanly(pm_lib):
    """In a container without a GPU the handle is not created and a CUDA status comes back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from probabilistic_mapping_b200 import _lib
    c = _lib.default_config(64, 48, 64)
    h = ctypes.c_void_p()
    assert pm_lib.pm_create(ctypes.byref(c), ctypes.byref(h)) == _lib.PM_ERR_CUDA
    assert not h.value


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from probabilistic_mapping_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libpm_stereo.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()


def test_checked_build_exports_the_same_entry_points(pm_lib):
    """libpm_stereo_checked.so (PM_BOUNDS_CHECK) is built beside the product library and exports
    the same C ABI; only the product library answers pm_debug_bounds with PM_ERR_UNSUPPORTED, and
    it does so without touching the GPU."""
    from probabilistic_mapping_b200 import _lib, build
    assert os.path.exists(build.LIB_CHECKED)
    checked = ctypes.CDLL(build.LIB_CHECKED)
    for n in declared():
        assert hasattr(checked, n), f"{n} missing from the checked build"
    out = (ctypes.c_uint64 * 4)(1, 2, 3, 4)
    assert pm_lib.pm_debug_bounds(out, 0) == _lib.PM_ERR_UNSUPPORTED and list(out) == [0, 0, 0, 0]
