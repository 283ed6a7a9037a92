import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "embree-benchmark-protoray_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_kats.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libprt_b200.so")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def small():
    import scenes
    mesh, view = scenes.small_scene()
    return mesh, view


@pytest.fixture(scope="session")
def small_path(tmp_path_factory, small):
    import scenes
    d = tmp_path_factory.mktemp("scenes")
    return scenes.write_scene(str(d), "small", small[0], small[1])


@pytest.fixture(scope="session")
def small_oracle(small, oracle_mod):
    mesh, _ = small
    return oracle_mod.Oracle().scene(mesh.positions, mesh.indices)
