"""Shared pytest setup.

* registers the ``gpu`` marker (tests that need a CUDA device);
* puts the repository root on ``sys.path`` so ``oracle`` (test infrastructure)
  and ``__graft_entry__`` import;
* loads the product package from ``cuckoo-filter_b200/`` under the module name
  ``cuckoo_b200`` (the directory name is not a Python identifier).
"""
from __future__ import annotations

import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
PKG_DIR = os.path.join(ROOT, "cuckoo-filter_b200")


def load_package():
    if "cuckoo_b200" in sys.modules:
        return sys.modules["cuckoo_b200"]
    spec = importlib.util.spec_from_file_location("cuckoo_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cuckoo_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def cfb():
    """The product package (cuckoo-filter_b200), with its library built."""
    import subprocess

    lib = os.path.join(PKG_DIR, "lib", "libcuckoo_b200.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(PKG_DIR, "build.py")], check=True)
    return load_package()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    return dict(np.load(os.path.join(ROOT, "tests", "golden", "candidates.npz")))


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.lib()
    return oracle
