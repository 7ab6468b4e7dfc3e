"""Shared fixtures: the libpt binding (package loaded by path), scene
generators, the CPU oracle and, where built, the reference shader code
compiled for the CPU."""

from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "pbrt-renderer-_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_package():
    """Import pbrt-renderer-_b200/ as module `pbrt_b200` (its directory name is
    not a Python identifier)."""
    if "pbrt_b200" in sys.modules:
        return sys.modules["pbrt_b200"]
    spec = importlib.util.spec_from_file_location("pbrt_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pbrt_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libpt.so")


@pytest.fixture(scope="session")
def pt():
    return load_package()


@pytest.fixture(scope="session")
def scenes(pt):
    return importlib.import_module("pbrt_b200.scenes")


@pytest.fixture(scope="session")
def oracle(pt):
    from oracle.oracle import Oracle
    return Oracle(pt)


@pytest.fixture(scope="session")
def reference(pt):
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference shader build (oracle/_ref/libref.so) not present")
    return Reference(pt)


@pytest.fixture(scope="session")
def ctx(pt):
    """A libpt context on cuda:0 (GPU tests only)."""
    c = pt.Context(0)
    yield c
    c.close()


def rel_err(a, b, floor):
    """|a - b| / max(|b|, floor), elementwise."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)
