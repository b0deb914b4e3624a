"""Shared test fixtures: loads the product package (``swl_b200``) and the oracle."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "seiswavelab--curvilinear_b200"
ORACLE_DIR = ROOT / "oracle"
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def load_package():
    """Import the product package (directory name is not a Python identifier)."""
    if "swl_b200" in sys.modules:
        return sys.modules["swl_b200"]
    spec = importlib.util.spec_from_file_location("swl_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["swl_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if str(ORACLE_DIR) not in sys.path:
        sys.path.insert(0, str(ORACLE_DIR))
    import oracle  # noqa: E402

    return oracle


@pytest.fixture(scope="session")
def swl():
    return load_package()


@pytest.fixture(scope="session")
def oracle_mod():
    return load_oracle()


@pytest.fixture(scope="session")
def orc(oracle_mod):
    return oracle_mod.Oracle()


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def has_reference_binaries(oracle_mod) -> bool:
    return oracle_mod.REF2D.exists() and oracle_mod.REF3D.exists()
