"""Shared test set-up: the ``gpu`` marker, the package and the checkers.

The package directory is ``licom3-hip_b200`` (not an identifier), so it is
loaded by path.  CPU-only tests never launch device work; tests marked
``gpu`` need a CUDA device and call the library through its C ABI.
"""
import importlib.util
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(REPO, "licom3-hip_b200")
sys.path.insert(0, os.path.join(REPO, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    lib = os.path.join(PKG_DIR, "liblicom_tracer.so")
    oracle = os.path.join(REPO, "oracle", "liblicom_oracle.so")
    if not os.path.exists(lib) or not os.path.exists(oracle):
        spec = importlib.util.spec_from_file_location("lt_build", os.path.join(PKG_DIR, "build.py"))
        b = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(b)
        if not os.path.exists(lib):
            b.build_cuda()
        if not os.path.exists(oracle):
            b.build_oracle()


def load_package():
    if "licom3_hip_b200" in sys.modules:
        return sys.modules["licom3_hip_b200"]
    _ensure_built()
    spec = importlib.util.spec_from_file_location(
        "licom3_hip_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["licom3_hip_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def lt():
    return load_package()


@pytest.fixture(scope="session")
def has_gpu(lt):
    return lt.device_count() > 0


@pytest.fixture(autouse=True)
def _skip_without_gpu(request):
    if request.node.get_closest_marker("gpu"):
        pkg = load_package()
        if pkg.device_count() == 0:
            pytest.skip("no CUDA device")
