import importlib.util
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "radiativeviewfactor.jl_b200"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def load_pkg():
    """Import the package directory (not a Python identifier) as rvf_b200."""
    if "rvf_b200" in sys.modules:
        return sys.modules["rvf_b200"]
    spec = importlib.util.spec_from_file_location("rvf_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["rvf_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def rvf():
    return load_pkg()


@pytest.fixture(scope="session")
def orc():
    from oracle import pyoracle
    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def session(rvf):
    """One library session on cuda:0 for all GPU tests."""
    from importlib import import_module
    build = import_module("rvf_b200.build")
    build.build()
    s = rvf.Session(0)
    yield s
    s.close()
