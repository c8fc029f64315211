import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200) and the built libqpb.so")


def gpu_present() -> bool:
    try:
        from qoraphasecu_b200 import _lib

        return bool(_lib.load().qpb_cuda_available())
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """Fails (does not skip) a GPU test that runs without a device or the library."""
    from qoraphasecu_b200 import _lib

    lib = _lib.load()
    assert lib.qpb_cuda_available(), "gpu test run without a CUDA device"
    return lib


@pytest.fixture(scope="session")
def readme():
    from synthetic import readme_triangle

    return readme_triangle()


os.environ.setdefault("OMP_NUM_THREADS", str(len(os.sched_getaffinity(0))))
