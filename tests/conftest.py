"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_bfb():
    """Import the product package (directory biofvm-b_b200) by path."""
    if "biofvm_b_b200" in sys.modules:
        return sys.modules["biofvm_b_b200"]
    pkg = ROOT / "biofvm-b_b200"
    spec = importlib.util.spec_from_file_location("biofvm_b_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["biofvm_b_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def bfb():
    return load_bfb()


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture
def rng():
    return np.random.default_rng(12345)


def log_uniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))
