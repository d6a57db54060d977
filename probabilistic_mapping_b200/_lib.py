"""ctypes binding of libpm_stereo.so (include/pm_stereo.h).

The library is built in-tree by probabilistic_mapping_b200/build.py.  There is no fallback:
if the shared library is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# PM_STEREO_LIB selects another build of the library (the bounds-checked libpm_stereo_checked.so)
LIB_PATH = os.environ.get("PM_STEREO_LIB") or os.path.join(HERE, "libpm_stereo.so")

PM_OK = 0
PM_ERR_INVALID_ARGUMENT = 1
PM_ERR_BAD_STATE = 2
PM_ERR_CUDA = 3
PM_ERR_OUT_OF_MEMORY = 4
PM_ERR_UNSUPPORTED = 5

PM_COST_REFERENCE = 0
PM_COST_CORRECTED = 1
PM_PREC_FP32 = 0
PM_PREC_FP16 = 1
PM_SAMPLER_EXACT = 0
PM_SAMPLER_TEXTURE = 1
PM_SAMPLER_TEXTURE_F32 = 2
PM_BATCH_HOST_IO = 1
PM_BATCH_AUTOTUNE = 2
PM_BATCH_PRIORITY = 4
PM_BATCH_PERSISTENT = 8
PM_BATCH_STATS = 16
PM_FUSION_GPU = 0
PM_FUSION_CPU_PATH = 1
PM_CASE_RAW_ARGMIN = 0
PM_CASE_SGM_ARGMIN = 1
PM_CASE_FILTERED = 2


class PmConfig(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("num_planes", ctypes.c_int),
        ("rho0", ctypes.c_float), ("rho_step", ctypes.c_float), ("intensity_scale", ctypes.c_float),
        ("num_paths", ctypes.c_int),
        ("p1", ctypes.c_float), ("p2", ctypes.c_float), ("tau_so", ctypes.c_float),
        ("q1", ctypes.c_float), ("q2", ctypes.c_float), ("var_scale", ctypes.c_float),
        ("uniqueness_ratio", ctypes.c_float),
        ("cost_mode", ctypes.c_int), ("precision", ctypes.c_int), ("fusion_variant", ctypes.c_int),
        ("tree_compat", ctypes.c_int), ("max_sources", ctypes.c_int), ("device", ctypes.c_int),
        ("sampler", ctypes.c_int),
    ]


class PmDiffConfig(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("num_planes", ctypes.c_int),
        ("num_sources", ctypes.c_int), ("rho0", ctypes.c_float), ("rho_step", ctypes.c_float),
        ("temperature", ctypes.c_float), ("p1", ctypes.c_float), ("p2", ctypes.c_float),
        ("tau_so", ctypes.c_float), ("q1", ctypes.c_float), ("q2", ctypes.c_float),
        ("store_paths", ctypes.c_int), ("device", ctypes.c_int),
    ]


class PmBuffers(ctypes.Structure):
    _fields_ = [("cost", ctypes.c_void_p), ("sgm", ctypes.c_void_p), ("wta_index", ctypes.c_void_p),
                ("wta_depth", ctypes.c_void_p), ("table", ctypes.c_void_p), ("cost_offset", ctypes.c_void_p)]


# pm_stats, in the order of its fields (include/pm_stereo.h)
STATS_FIELDS = ("wta_depth", "wta_no_overlap", "wta_border", "wta_flat", "wta_ambiguous",
                "tf_empty", "tf_outlier", "tf_behind", "tf_outside", "tf_moved",
                "pred_none", "pred_copied", "pred_filled",
                "upd_empty", "upd_init", "upd_no_measurement", "upd_output", "upd_hidden")


class PmStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in STATS_FIELDS]


# Every exported entry point with its argument types; also the list the load test checks.
_P, _VP, _SZ, _I, _F = ctypes.POINTER, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_float
_D = _P(ctypes.c_double)
SIGNATURES = {
    "pm_config_default": (None, [_P(PmConfig), _I, _I, _I]),
    "pm_create": (_I, [_P(PmConfig), _P(_VP)]),
    "pm_destroy": (None, [_VP]),
    "pm_set_stream": (_I, [_VP, _VP]),
    "pm_init_intrinsic": (_I, [_VP, _D, _F, _F]),
    "pm_init_reference": (_I, [_VP, _VP, _SZ]),
    "pm_update": (_I, [_VP, _VP, _SZ, _D, _D, _D, _D]),
    "pm_output": (_I, [_VP, _VP, _SZ]),
    "pm_output_fusion": (_I, [_VP, _VP, _SZ, _VP, _SZ, _D, _D, _F, _F, _F, _F]),
    "pm_output_case": (_I, [_VP, _I, _VP, _SZ]),
    "pm_get_wta_depth": (_I, [_VP, _VP, _SZ]),
    "pm_get_wta_index": (_I, [_VP, _VP]),
    "pm_get_state": (_I, [_VP, _VP, _VP, _VP, _VP]),
    "pm_set_state": (_I, [_VP, _VP, _VP, _VP, _VP, _D, _D]),
    "pm_get_buffers": (_I, [_VP, _P(PmBuffers)]),
    "pm_debug_store_sgm": (_I, [_VP, _I]),
    "pm_get_homography": (_I, [_VP, _I, _P(ctypes.c_float)]),
    "pm_enable_stage_timing": (_I, [_VP, _I]),
    "pm_get_stage_times": (_I, [_VP, _P(ctypes.c_float), _I]),
    "pm_enable_stats": (_I, [_VP, _I]),
    "pm_get_stats": (_I, [_VP, _P(PmStats)]),
    "pm_synchronize": (_I, [_VP]),
    "pm_debug_check_arith": (_I, [_P(ctypes.c_uint64), _VP]),
    "pm_debug_bounds": (_I, [_P(ctypes.c_uint64), _I]),
    "pm_last_error": (ctypes.c_char_p, [_VP]),
    "pm_status_string": (ctypes.c_char_p, [_I]),
    "pm_stage_to_float": (_I, [_I, _I, _VP, _SZ, _VP, _F, _VP]),
    "pm_stage_calc_cost": (_I, [_P(PmConfig), _VP, _VP, _I, _P(ctypes.c_float), _VP, _VP, _VP, _VP]),
    "pm_stage_sgm": (_I, [_P(PmConfig), _VP, _VP, _VP, _VP, _VP]),
    "pm_stage_filter": (_I, [_P(PmConfig), _VP, _VP, _SZ, _VP, _VP]),
    "pm_stage_sgm_filter": (_I, [_P(PmConfig), _VP, _VP, _VP, _VP, _SZ, _VP, _VP]),
    "pm_stage_depth_fuse": (_I, [_I, _I, _P(ctypes.c_float), _P(ctypes.c_float), _VP, _P(_VP), _P(_VP),
                                 _VP, _VP, _VP]),
    "pm_stage_convert": (_I, [_I, _I, _VP, _VP, _I, _SZ, _VP]),
    "pm_stage_depth_fuse_noalloc": (_I, [_I, _I, _P(ctypes.c_float), _P(ctypes.c_float), _VP, _P(_VP),
                                         _P(_VP), _VP, _VP]),
    "pm_batch_create": (_I, [_P(PmConfig), _I, _I, _I, _I, _P(_VP)]),
    "pm_batch_destroy": (None, [_VP]),
    "pm_batch_init_intrinsic": (_I, [_VP, _I, _D, _F]),
    "pm_batch_frame": (_I, [_VP, _I, _I, _P(_VP)]),
    "pm_batch_put_frame": (_I, [_VP, _I, _I, _VP, _SZ]),
    "pm_batch_set_poses": (_I, [_VP, _I, _D, _D, _D, _D]),
    "pm_batch_run": (_I, [_VP]),
    "pm_batch_synchronize": (_I, [_VP]),
    "pm_batch_output": (_I, [_VP, _I, _P(_VP), _P(_VP)]),
    "pm_batch_copy_output": (_I, [_VP, _I, _VP, _SZ, _VP, _SZ]),
    "pm_batch_wta_depth": (_I, [_VP, _I, _P(_VP)]),
    "pm_batch_copy_wta_depth": (_I, [_VP, _I, _VP, _SZ]),
    "pm_stage_depth_fuse_cpu_path_scratch": (_SZ, [_I, _I]),
    "pm_stage_depth_fuse_cpu_path": (_I, [_I, _I, _P(ctypes.c_double), _P(ctypes.c_float), _VP, _P(_VP), _P(_VP),
                                          _VP, _VP, _VP]),
    "pm_batch_tuning": (_I, [_VP, _I, _P(_I), _P(_I), _P(_F)]),
    "pm_batch_get_stats": (_I, [_VP, _I, _P(PmStats)]),
    "pm_batch_stream": (_VP, [_VP]),
    "pm_batch_last_error": (ctypes.c_char_p, [_VP]),
    "pm_diff_config_default": (None, [_P(PmDiffConfig), _I, _I, _I, _I]),
    "pm_diff_create": (_I, [_P(PmDiffConfig), _P(_VP)]),
    "pm_diff_destroy": (None, [_VP]),
    "pm_diff_memory": (_I, [_VP, _P(_SZ)]),
    "pm_diff_forward": (_I, [_VP, _VP, _VP, _D, _D, _D, _VP, _VP, _D, _VP]),
    "pm_diff_backward": (_I, [_VP, _VP, _D, _VP]),
    "pm_diff_last_error": (ctypes.c_char_p, [_VP]),
    "pm_pyr_down_u8": (_I, [_I, _I, _VP, _SZ, _VP, _SZ, _VP]),
    "pm_depth_up2": (_I, [_I, _I, _VP, _SZ, _VP, _SZ, _VP]),
    "pm_depth_range_mask": (_I, [_I, _I, _VP, _SZ, _F, _F, _VP]),
    "pm_colorize_depth": (_I, [_I, _I, _VP, _SZ, _VP, _SZ, _VP, _SZ, _VP, _VP]),
    "pm_write_pfm": (_I, [ctypes.c_char_p, _I, _I, _VP, _SZ]),
    "pm_write_npy": (_I, [ctypes.c_char_p, _I, _I, _VP, _SZ]),
    "pm_write_ppm": (_I, [ctypes.c_char_p, _I, _I, _VP, _SZ]),
    "pm_read_image_u8": (_I, [ctypes.c_char_p, _P(_I), _P(_I), _VP, _SZ]),
}

_lib = None


class PmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


def load():
    """Load libpm_stereo.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run probabilistic_mapping_b200/build.py "
                               "(the CUDA library is required; there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int, handle=None, what: str = "") -> None:
    if status != PM_OK:
        lib = load()
        msg = lib.pm_status_string(status).decode()
        if handle is not None:
            detail = lib.pm_last_error(handle)
            if detail:
                msg += ": " + detail.decode()
        raise PmError(status, f"{what}: {msg}" if what else msg)


def default_config(width: int, height: int, num_planes: int) -> PmConfig:
    cfg = PmConfig()
    load().pm_config_default(ctypes.byref(cfg), width, height, num_planes)
    return cfg
