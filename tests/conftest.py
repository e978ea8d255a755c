"""Shared test setup: markers, paths and loaders for the package, the oracle and goldens."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "oracle"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built engine")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def lv():
    """The engine package (directory name is not an identifier, so import by string)."""
    return importlib.import_module("louvain-fast-move-cuda_b200")


@pytest.fixture(scope="session")
def graphs():
    return importlib.import_module("louvain-fast-move-cuda_b200.graphs")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def golden():
    import make_golden
    return make_golden
