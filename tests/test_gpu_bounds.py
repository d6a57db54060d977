"""The bounds-checked build (libpm_stereo_checked.so, PM_BOUNDS_CHECK) on odd image shapes and
64 to 256 planes: every
checked global access of the cost, rebase, SGM pair, combine, counting and fusion kernels stays
inside its buffer (the record of skipped accesses is empty), and the checked build's outputs are
bit-identical to the product library's on the same inputs.  Both libraries run the same workload
(tests/bounds_workload.py) in child processes, one library per process."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def run(lib, path):
    env = dict(os.environ, PM_STEREO_LIB=lib)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "bounds_workload.py"), str(path)],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.load(path)


def test_checked_build_stays_in_bounds_and_matches_product(pm_lib, tmp_path):
    from probabilistic_mapping_b200 import _lib, build
    checked = run(build.LIB_CHECKED, tmp_path / "checked.npz")
    product = run(build.LIB, tmp_path / "product.npz")
    assert int(checked["bounds_status"][0]) == _lib.PM_OK
    assert int(product["bounds_status"][0]) == _lib.PM_ERR_UNSUPPORTED
    assert int(checked["bounds"][0]) == 0, f"out-of-range accesses: site, index, extent = {checked['bounds'][1:]}"
    keys = [k for k in product.files if not k.startswith("bounds")]
    assert len(keys) > 50 and set(keys) == set(k for k in checked.files if not k.startswith("bounds"))
    for k in keys:
        a, b = product[k], checked[k]
        assert a.shape == b.shape and (a.view(np.uint8) == b.view(np.uint8)).all(), k
