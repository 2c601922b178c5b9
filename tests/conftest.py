"""Shared fixtures: the product package (loaded by path, its directory name has a hyphen) and the
oracle. GPU tests carry @pytest.mark.gpu; everything else runs on a CPU-only machine."""
import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "hashjoin-scm_b200"


def load_package():
    if "hashjoin_scm_b200" in sys.modules:
        return sys.modules["hashjoin_scm_b200"]
    spec = importlib.util.spec_from_file_location("hashjoin_scm_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hashjoin_scm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if "hj_oracle" in sys.modules:
        return sys.modules["hj_oracle"]
    spec = importlib.util.spec_from_file_location("hj_oracle", ROOT / "oracle" / "hj_oracle.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hj_oracle"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def hj():
    mod = load_package()
    if not mod.LIB_PATH.exists():
        mod.build()
    mod.lib()
    return mod


@pytest.fixture(scope="session")
def oracle():
    mod = load_oracle()
    mod.lib()
    return mod


@pytest.fixture(scope="session")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
