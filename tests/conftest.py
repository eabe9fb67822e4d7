"""Shared fixtures; registers the `gpu` marker for tests that need a B200."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def nb():
    """The backend package (builds the CUDA library in place if needed)."""
    build = importlib.import_module("necsim-rust_b200.build")
    build.build()
    return importlib.import_module("necsim-rust_b200")


@pytest.fixture(scope="session")
def syn():
    return importlib.import_module("necsim-rust_b200.synthetic")


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.build()
    return o


@pytest.fixture(scope="session")
def kat():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "kat.json")) as f:
        return json.load(f)
