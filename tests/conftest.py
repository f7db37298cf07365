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


@pytest.fixture(scope="session", autouse=True)
def bounds_record():
    """With MPX_BOUNDS_CHECK_RUN=1 (set by tests/test_gpu_bounds.py together
    with MPX_LIBRARY=libmpx_checked.so): after the session, the checked
    library must report that no per-cell field access was out of range."""
    yield
    if os.environ.get("MPX_BOUNDS_CHECK_RUN") != "1":
        return
    import ctypes

    import mumaxplus_b200

    lib = mumaxplus_b200._abi.load()
    bad = ctypes.c_ulonglong(0)
    st = lib.mpx_bounds_check(ctypes.byref(bad))
    assert st == 0, f"mpx_bounds_check: status {st} ({lib.mpx_last_error()}); not the checked build?"
    v = bad.value
    assert v == 0, f"out-of-range field access: index {v & 0xFFFFFFFF} with N = {(v >> 32) & 0x7FFFFFFF}"
