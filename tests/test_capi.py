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


def test_cpp_drop_in_header_compiles(tmp_path):
    # the C++ drop-in layer (Kernel<T>, Tensor<T,N> with get_local_block and the block
    # iterators, BlockSpan) compiles and links against the library; it runs under -m gpu
    import subprocess
    exe = tmp_path / "drop_in"
    libdir = os.path.dirname(sht.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "drop_in.cpp"), "-L", libdir, "-lshtensor_b200",
           f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
