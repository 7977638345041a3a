"""Shared pytest setup: the `gpu` marker and fixtures for the B200 tests."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built library")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def native():
    """The C-ABI binding; on a GPU run the library must be built and load."""
    from gpumetropolis_b200 import _native
    from gpumetropolis_b200.build import build
    build()
    _native.load()
    return _native


@pytest.fixture(scope="session")
def gpu(native):
    if not native.available():
        pytest.fail("gpu test on a machine without a usable sm_100 device")
    return native
