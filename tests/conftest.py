"""Shared test setup: loads the engine package (its directory name is not a Python
identifier, so it is registered as `piv_b200`) and registers the `gpu` marker."""
import importlib.util
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "piv_xcorr2d_v1.0_b200"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def _load_pkg():
    if "piv_b200" in sys.modules:
        return sys.modules["piv_b200"]
    spec = importlib.util.spec_from_file_location("piv_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["piv_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_pkg()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA engine")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def pkg():
    return _load_pkg()


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")
    return True
