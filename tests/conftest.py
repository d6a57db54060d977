import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libpm_stereo.so")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this container")
    for it in items:
        if it.get_closest_marker("gpu") is not None:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def pm_lib():
    from probabilistic_mapping_b200 import build
    build.build()
    from probabilistic_mapping_b200 import _lib
    return _lib.load()


def small_case(W=96, H=64, D=64, S=3, seed=3, f=None, mode=0, paths=8, uniq=0.95, scale=1 / 255):
    """A seeded synthetic frame set with bench-style parameters, shared by several tests."""
    import oracle
    from probabilistic_mapping_b200 import scene
    f = f if f is not None else 0.8 * W
    fs = scene.make_frameset(W, H, f, S, seed=seed)
    rho0, drho = scene.plane_range(D)
    p = oracle.Params(W=W, H=H, D=D, drho=drho, rho0=rho0, intensity_scale=scale, cost_mode=mode,
                      num_paths=paths, p1=0.003, p2=0.01, tau_so=3.5 / 255, uniqueness=uniq)
    return fs, p


def homographies(fs):
    import oracle
    return np.stack([oracle.compose_homography(fs.K, fs.R_ref, fs.T_ref, fs.R_srcs[s], fs.T_srcs[s])
                     for s in range(fs.srcs.shape[0])])
