"""Shared test set-up: the `gpu` marker, the package loader, oracle fixtures."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_DIR = os.path.join(ROOT, "earthquakediffinitive.jl_b200")


def load_package():
    """Import the `earthquakediffinitive.jl_b200` directory as `eqd_b200`."""
    if "eqd_b200" in sys.modules:
        return sys.modules["eqd_b200"]
    spec = importlib.util.spec_from_file_location(
        "eqd_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["eqd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libeqd.so")


@pytest.fixture(scope="session")
def eqd():
    return load_package()
