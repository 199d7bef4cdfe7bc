"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device")


@pytest.fixture(scope="session")
def ge():
    """The product package (directory name has a hyphen: import by name)."""
    return importlib.import_module("galaxy-engine_b200")


@pytest.fixture(scope="session")
def ics():
    return importlib.import_module("galaxy-engine_b200.ics")


@pytest.fixture(scope="session")
def O():
    import oracle
    return oracle


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
