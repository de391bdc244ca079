"""The C-ABI library loads and exports every entry point include/shtensor_b200.h declares
(CPU-only: no compute calls)."""
import ctypes
import os
import re

import pytest

import shtensor_b200 as sht

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "shtensor_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sht_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(sht.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert sorted(set(sht.exported_symbols())) == declared_symbols()


def test_no_gpu_fails_loudly():
    from tests.conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sht.ShtError) as ei:
        sht.Context(1 << 20)
    assert ei.value.status in (sht.Status.ERR_CUDA, sht.Status.ERR_OOM)
