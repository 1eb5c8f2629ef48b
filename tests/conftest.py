import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
os.environ.setdefault("PPCB_QUIET", "1")

ICE_CACHE = os.path.join(ROOT, "ppc_b200", "data", "ice")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _ice(kind):
    from ppc_b200 import synth
    path = os.path.join(ICE_CACHE, kind)
    if not os.path.exists(os.path.join(path, "cfg.txt")):
        synth.write(kind, path)
    return path


@pytest.fixture(scope="session")
def ice_small():
    return _ice("small")


@pytest.fixture(scope="session")
def ice_full():
    return _ice("full")


@pytest.fixture(scope="session")
def ice_full2d():
    return _ice("full2d")


@pytest.fixture(scope="session")
def ice_small_xr1():
    return _ice("small_xr1")


@pytest.fixture(scope="session")
def ice_full_ng():
    return _ice("full_ng")


@pytest.fixture(scope="session")
def ice_small_tilt():
    return _ice("small_tilt")


@pytest.fixture(scope="session")
def ice_small_hole():
    return _ice("small_hole")


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
