"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and run on a B200;
everything else runs on the CPU (oracle, host logic, C-ABI surface)."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "explicit-gpumpm-ductile-fracture_b200"
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_package():
    if "gmpm_b200" in sys.modules:
        return sys.modules["gmpm_b200"]
    spec = importlib.util.spec_from_file_location("gmpm_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gmpm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    # Build the library in-tree if needed (nvcc cross-compiles without a GPU).
    spec = importlib.util.spec_from_file_location("gmpm_build", PKG_DIR / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build()
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O  # oracle/oracle.py
    O.build()
    return O


@pytest.fixture(scope="session")
def ctx(pkg):
    c = pkg.gmpm.Context(0)
    yield c
    c.close()
