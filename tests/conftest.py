"""Test setup: the `gpu` marker, the package import and the oracle path.

The package directory is named `spuma-multiphysics_b200`; it is registered here
as the importable module `spuma_multiphysics_b200`.
"""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def _register_package():
    name = "spuma_multiphysics_b200"
    if name in sys.modules:
        return
    pkg_dir = ROOT / "spuma-multiphysics_b200"
    spec = importlib.util.spec_from_file_location(name, pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    module = importlib.util.module_from_spec(spec)
    sys.modules[name] = module
    spec.loader.exec_module(module)


_register_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda_available():
    import torch
    return torch.cuda.is_available()
