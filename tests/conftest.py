"""Test configuration: the `gpu` marker and package loading.

The package directory is named ``oxideav-av1_b200`` (not an importable
identifier), so it is registered under the module name ``oxideav_av1_b200``.
"""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "oxideav-av1_b200"


def load_package():
    if "oxideav_av1_b200" in sys.modules:
        return sys.modules["oxideav_av1_b200"]
    spec = importlib.util.spec_from_file_location("oxideav_av1_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["oxideav_av1_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
