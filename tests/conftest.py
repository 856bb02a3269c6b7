"""Shared test setup: loads the package directory `lastz-gxy_b200` as
`lastz_gxy_b200`, puts the oracle on the path, and registers the `gpu` marker."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load_pkg():
    if "lastz_gxy_b200" in sys.modules:
        return sys.modules["lastz_gxy_b200"]
    pkg_dir = os.path.join(ROOT, "lastz-gxy_b200")
    spec = importlib.util.spec_from_file_location("lastz_gxy_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lastz_gxy_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_pkg()
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gxy():
    return sys.modules["lastz_gxy_b200"]


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def ctx(gxy):
    return gxy.Context.default(0)
