import importlib.util
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_pp():
    """Import the package directory `pastel-palettes_b200` as `pastel_palettes_b200`."""
    if "pastel_palettes_b200" in sys.modules:
        return sys.modules["pastel_palettes_b200"]
    pkg = os.path.join(ROOT, "pastel-palettes_b200")
    if not os.path.exists(os.path.join(pkg, "libpastel_palettes.so")):
        subprocess.run(["make", "-C", os.path.join(pkg, "csrc")], check=True, stdout=subprocess.DEVNULL)
    spec = importlib.util.spec_from_file_location("pastel_palettes_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pastel_palettes_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pp():
    return load_pp()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.lib()
    return o


@pytest.fixture(scope="session")
def hctx(pp):
    """Host-only planning context (no device)."""
    return pp.Context(device=-1)


@pytest.fixture(scope="session")
def gctx(pp):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return pp.Context(device=0)
