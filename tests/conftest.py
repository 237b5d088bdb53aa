"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _load_pkg():
    name = "pe_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, ROOT / "protein_encoding_v2_nsga-iii_b200" / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_pkg_module(stem):
    """A pure-Python module of the package (server, replicas) under the name pe_b200_<stem>."""
    name = f"pe_b200_{stem}"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, ROOT / "protein_encoding_v2_nsga-iii_b200" / f"{stem}.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pe():
    return _load_pkg()


@pytest.fixture(scope="session")
def orc():
    import pe_oracle
    pe_oracle.lib()
    return pe_oracle


@pytest.fixture(scope="session")
def ref_table(pe):
    return pe.load_codon_table(ROOT / "protein_encoding_v2_nsga-iii_b200" / "data" / "ref_codon_table.txt")


@pytest.fixture(scope="session")
def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu(cuda_ok):
    if not cuda_ok:
        pytest.fail("GPU test collected without a CUDA device")
    return True
