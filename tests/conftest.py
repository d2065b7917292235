"""Test setup: registers the ``gpu`` marker and loads the package (its
directory name is not a Python identifier) under the name ``feicar_b200``."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "feicar3d_3.0_febio_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def _load_pkg():
    if "feicar_b200" in sys.modules:
        return sys.modules["feicar_b200"]
    spec = importlib.util.spec_from_file_location(
        "feicar_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR]
    )
    mod = importlib.util.module_from_spec(spec)
    sys.modules["feicar_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_pkg()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: CPU test that takes more than a few seconds")
