import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_NAME = "b-tree-index-searching_b200"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device")


def load_pkg():
    """The engine's Python binding package (directory name has dashes)."""
    return importlib.import_module(PKG_NAME)


def load_workloads():
    return importlib.import_module(PKG_NAME + ".workloads")


@pytest.fixture(scope="session")
def bt():
    return load_pkg()


@pytest.fixture(scope="session")
def wl():
    return load_workloads()


@pytest.fixture(scope="session")
def orc():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
