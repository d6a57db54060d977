"""The FP32 kernels replace IEEE operations by cheaper sequences that must give the same bits (a
Newton step from the hardware reciprocal, an add-based floor, a reciprocal-multiply division by
a small integer) or follow a stated rule (the branch-free reciprocal of the warps, which the FP32
oracle implements too).  This re-runs the exhaustive device-side comparison."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_exact_arithmetic_shortcuts(pm_lib):
    out = (ctypes.c_uint64 * 4)()
    assert pm_lib.pm_debug_check_arith(out, None) == 0
    assert list(out) == [0, 0, 0, 0], f"mismatches: rcp={out[0]} floor={out[1]} div={out[2]} warp rcp={out[3]}"
