"""The C++ drop-in layer (include/shtensor_b200.hpp): a program written like the reference's
own tests compiles against it, links the CUDA library and passes on the B200."""
import os
import subprocess

import pytest

import shtensor_b200 as sht

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_drop_in(tmp_path):
    exe = tmp_path / "drop_in"
    libdir = os.path.dirname(sht.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "drop_in.cpp"),
           "-L", libdir, "-lshtensor_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
