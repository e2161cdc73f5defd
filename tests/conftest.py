import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


def _have_gpu() -> bool:
    try:
        import ctypes
        lib = ctypes.CDLL("libcuda.so.1")
        n = ctypes.c_int(0)
        if lib.cuInit(0) != 0:
            return False
        return lib.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


HAVE_GPU = _have_gpu()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def _build_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("legendre_b200_build", ROOT / "legendre_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# build before any test module imports the package (a stale library would
# miss symbols); cheap when up to date
_build_module().build_library()
_build_module().build_oracle()


@pytest.fixture(scope="session")
def orc():
    import oracle_bind
    return oracle_bind


@pytest.fixture(scope="session")
def sched():
    from legendre_b200 import CudaScheduler
    s = CudaScheduler(0)
    yield s
    s.close()
