"""Shared test setup: the `gpu` marker, loaders for the package (swd_b200) and the
oracle, and small helpers.  Tests marked gpu need a CUDA device; everything else runs on
the CPU.  The oracle (oracle/) is only ever used here as the checker."""
import importlib.util
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "simple-wavenumber-deconvolution_b200"
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT / "oracle"))


def load_pkg():
    if "swd_b200" in sys.modules:
        return sys.modules["swd_b200"]
    spec = importlib.util.spec_from_file_location("swd_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["swd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="session")
def swd():
    return load_pkg()


@pytest.fixture(scope="session")
def orc():
    import pyoracle
    pyoracle.lib()
    return pyoracle
