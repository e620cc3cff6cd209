import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "aocl-data-analytics_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ab():
    """The ctypes binding of libaoclda_b200.so (built in-tree)."""
    lib = os.path.join(PKG, "libaoclda_b200.so")
    if not os.path.exists(lib):
        import subprocess
        subprocess.run(["make", "-s", "-j8", "-C", PKG], check=True)
    return _load("aoclda_b200", os.path.join(PKG, "aoclda_b200.py"))


@pytest.fixture(scope="session")
def orc():
    """The CPU oracle (test infrastructure)."""
    return _load("oracle_mod", os.path.join(ORACLE, "oracle.py"))


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return True


def golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def da(ab):
    """The ``aoclda`` drop-in Python package (aocl-data-analytics_b200/python)."""
    path = os.path.join(PKG, "python")
    if path not in sys.path:
        sys.path.insert(0, path)
    import aoclda
    import aoclda.faiss
    import aoclda.metrics
    import aoclda.sklearn
    return aoclda
