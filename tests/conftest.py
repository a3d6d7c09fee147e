"""Test configuration: the ``gpu`` marker and import paths.

The package directory is named ``ipeps.jl_b200`` (not an importable name), so
it is registered here as the module ``ipeps_b200``.  The CPU oracle lives in
``oracle/`` and is imported as ``ipeps_oracle`` (tests only).
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_package():
    if "ipeps_b200" in sys.modules:
        return sys.modules["ipeps_b200"]
    pkg_dir = os.path.join(ROOT, "ipeps.jl_b200")
    spec = importlib.util.spec_from_file_location("ipeps_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ipeps_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def engine(pkg):
    if not gpu_available():
        pytest.skip("no CUDA device")
    return pkg.Engine(0)
