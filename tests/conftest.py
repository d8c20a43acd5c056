"""pytest configuration: the `gpu` marker and loading of the library package.

The package directory is ``nflow-red-poplar_b200`` (not an importable name),
so it is loaded by path and registered as ``nflow_red_poplar_b200``.
"""
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_package():
    name = "nflow_red_poplar_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "nflow-red-poplar_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
