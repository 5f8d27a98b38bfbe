"""Test set-up: the `gpu` marker, and import helpers for the package (its
directory name has dashes, so it is loaded under the name `pcg`) and for
the oracle (test infrastructure under oracle/)."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "physicell-mac-metal_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_package():
    if "pcg" in sys.modules:
        return sys.modules["pcg"]
    spec = importlib.util.spec_from_file_location("pcg", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pcg"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libpcg.so")


@pytest.fixture(scope="session")
def pcg():
    return load_package()


@pytest.fixture(scope="session")
def po():
    import pyoracle
    return pyoracle


@pytest.fixture(scope="session")
def ctx(pcg):
    c = pcg.Context(0)
    yield c
    c.close()
