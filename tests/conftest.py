import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _have_gpu():
    try:
        import ctypes
        rt = None
        for name in ("libcuda.so.1", "libcuda.so"):
            try:
                rt = ctypes.CDLL(name)
                break
            except OSError:
                continue
        if rt is None:
            return False
        n = ctypes.c_int(0)
        if rt.cuInit(0) != 0:
            return False
        return rt.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def syn():
    import synergia2_b200
    return synergia2_b200


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    return O
