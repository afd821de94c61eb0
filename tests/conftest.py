import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "skirt9-gpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
    return load


@pytest.fixture
def oracle_backend():
    import oracle
    be = oracle.backend()
    yield be
    be.close()


@pytest.fixture
def gpu_backend():
    from skgpu import Backend
    be = Backend()  # raises if lib/libskgpu.so is missing or no device: no fallback
    yield be
    be.close()


PATH_FIXTURES = ["cartesian_selftest", "cartesian_c16", "octree", "voronoi", "tetra", "sphere1d", "cylinder2d", "sphere2d", "sphere3d", "cylinder3d", "adaptive"]


def segments_of(z, r):
    off = z["ray_offset"]
    return z["ray_m"][off[r]:off[r + 1]], z["ray_ds"][off[r]:off[r + 1]]
