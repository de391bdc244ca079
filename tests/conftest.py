"""Shared test setup.  CPU tests (-m "not gpu") check the oracle against the reference's own
headers and numpy, and that the C-ABI library loads; GPU tests (-m gpu) are the parity tests
proper and call the CUDA library through its C ABI."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       capture_output=True)


_ensure_oracle()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    import shtensor_b200 as sht
    c = sht.Context(8 << 30)
    yield c
    c.close()
