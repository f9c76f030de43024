import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "water-sim-cuda_b200")
for p in (PKG, ROOT, os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def reference_tree():
    """The reference's source tree (read as text by a few host tests when it
    is present): $MPM_REF_TREE, else BASELINE.json's `reference_path`."""
    import json
    env = os.environ.get("MPM_REF_TREE")
    if env:
        return env
    try:
        with open(os.path.join(ROOT, "BASELINE.json")) as f:
            return json.load(f).get("reference_path")
    except (OSError, ValueError):
        return None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU; run with -m gpu")


def pytest_collection_modifyitems(config, items):
    # Files named test_zz_* run after every other test file.
    items.sort(key=lambda it: os.path.basename(str(it.fspath)).startswith("test_zz_"))


@pytest.fixture(scope="session")
def oracle64():
    from oracle.oracle import Oracle
    return Oracle(64)


@pytest.fixture(scope="session")
def oracle32():
    from oracle.oracle import Oracle
    return Oracle(32)


@pytest.fixture(scope="session")
def mpm():
    import mpm_b200
    return mpm_b200


@pytest.fixture(scope="session")
def gpu_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected but no CUDA device is visible")
    return True
