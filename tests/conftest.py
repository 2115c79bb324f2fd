"""Shared fixtures: load the package from its directory and the oracle."""
import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "multiscale-and-multiphysics-integrated-simulator-for-tsunami_b200"


def load_pkg():
    if "cadmas_b200" in sys.modules:
        return sys.modules["cadmas_b200"]
    spec = importlib.util.spec_from_file_location("cadmas_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cadmas_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    try:
        import pyoracle
    finally:
        sys.path.pop(0)
    return pyoracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def orc():
    load_pkg()
    return load_oracle()


@pytest.fixture(scope="session")
def gpu_lib(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg.build_library()
    return pkg.load_library()
