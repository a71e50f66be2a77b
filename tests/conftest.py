import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")


def _has_gpu():
    try:
        import azimuth_b200
        return azimuth_b200.device_info(0) is not None
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.fail("GPU test selected but no CUDA device is usable")
    return True


@pytest.fixture(scope="session", autouse=True)
def built_library():
    """Build the native library (and the C oracle) once per session if stale."""
    from azimuth_b200 import build
    build.build()
    return True
