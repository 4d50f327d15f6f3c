"""Shared fixtures.  `gpu` marks tests that need a CUDA device (run with
`-m gpu`); everything else runs on the CPU."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_pkg():
    if "erebus_b200" in sys.modules:
        return sys.modules["erebus_b200"]
    pkg_dir = os.path.join(ROOT, "erebus.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "erebus_b200", os.path.join(pkg_dir, "__init__.py"),
        submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["erebus_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


@pytest.fixture(scope="session")
def oracle():
    load_pkg()
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def built_lib(pkg):
    from importlib import import_module
    build = import_module("erebus_b200.build")
    build.build()
    return pkg.load_library()
