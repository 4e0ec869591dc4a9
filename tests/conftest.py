"""Test configuration: the `gpu` marker and loaders for the package and the oracle.

The package directory is named lsdem2.0_b200, which is not an importable
module name, so it is loaded from its path under the module name lsdem_b200.
"""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "lsdem2.0_b200"


def load_package():
    if "lsdem_b200" in sys.modules:
        return sys.modules["lsdem_b200"]
    spec = importlib.util.spec_from_file_location("lsdem_b200", PKG / "__init__.py",
                                                  submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lsdem_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if str(ROOT / "oracle") not in sys.path:
        sys.path.insert(0, str(ROOT / "oracle"))
    import oracle  # noqa: E402
    return oracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def lsdem():
    return load_package()


@pytest.fixture(scope="session")
def ora():
    return load_oracle()
