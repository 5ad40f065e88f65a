"""Shared test setup: the `gpu` marker, the package loader and fixtures."""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def load_bolt():
    """Imports the package directory `craton-bolt_b200` as `craton_bolt_b200`."""
    name = "craton_bolt_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = REPO / "craton-bolt_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def bolt():
    return load_bolt()


@pytest.fixture(scope="session")
def engine(bolt):
    eng = bolt.Engine(0, scratch_bytes=6 << 30)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc
    orc.build()
    return orc
