import ctypes
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from equelle_b200 import capi  # noqa: E402

ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "libeqg_oracle.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libeqg.so")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    """The CPU oracle (test infrastructure only)."""
    if not os.path.exists(ORACLE_LIB):
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    return capi.bind(ctypes.CDLL(ORACLE_LIB, mode=ctypes.RTLD_LOCAL))


@pytest.fixture(scope="session")
def gpu_lib():
    """The device runtime; GPU tests fail (not skip) if it cannot load."""
    if not _cuda_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    import equelle_b200
    return equelle_b200.load_library()
