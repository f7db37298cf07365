import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libmpx.so")
    config.addinivalue_line("markers", "slow: long-running oracle check")


def gpu_available():
    try:
        import ctypes

        lib_path = os.path.join(ROOT, "mumax-plus_b200", "libmpx.so")
        if not os.path.exists(lib_path):
            return False
        lib = ctypes.CDLL(lib_path)
        return lib.mpx_device_count() > 0
    except OSError:
        return False


@pytest.fixture(scope="session")
def oracle():
    import oracle as _o

    _o.build()
    return _o


@pytest.fixture(scope="session")
def mpx():
    if not gpu_available():
        pytest.fail("GPU test needs a CUDA device and mumax-plus_b200/libmpx.so")
    import mumaxplus_b200

    return mumaxplus_b200
