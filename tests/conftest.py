"""pytest set-up: the `gpu` marker, and import paths for the package and the oracle.

The package directory is named `hype-parallel_b200` (not an importable
identifier), so it is loaded here under the module name `hype_parallel_b200`.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _load_package():
    if "hype_parallel_b200" in sys.modules:
        return sys.modules["hype_parallel_b200"]
    pkg_dir = os.path.join(ROOT, "hype-parallel_b200")
    spec = importlib.util.spec_from_file_location("hype_parallel_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hype_parallel_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) CUDA device")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def hp():
    return sys.modules["hype_parallel_b200"]


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.Oracle()
