"""Exact float forms of the reference's float-against-double compares used by the kernels.

The winner-take-all and the CASE argmin test |min| < FLOAT_EPS with FLOAT_EPS = 1e-5 as a double
(filter_cost.cu:37, parameters.h:6); the kernels compare in FP32 against kFloatEpsBelow
(csrc/sgm_device.cuh), which is exact when that constant is the largest float below 1e-5.
"""
import re

import numpy as np

from conftest import ROOT


def test_float_eps_bound_is_the_largest_float_below_1e_5():
    src = open(f"{ROOT}/probabilistic_mapping_b200/csrc/sgm_device.cuh").read()
    lit = re.search(r"constexpr float kFloatEpsBelow = ([0-9.e+-]+)f;", src).group(1)
    b = np.float32(float(lit))
    assert float(b) < 1e-5 <= float(np.nextafter(b, np.float32(np.inf)))
    # every float x: (double)x < 1e-5 exactly when x <= b, and (double)x > -1e-5 when x >= -b
    xs = np.array([b, np.nextafter(b, np.float32(1)), np.nextafter(b, np.float32(0)), np.float32(1e-5),
                   -b, np.float32(0), np.float32(-0.0), np.float32(2e-5)], np.float32)
    for x in xs:
        assert (float(x) < 1e-5) == (x <= b)
        assert (float(x) > -1e-5) == (x >= -b)
