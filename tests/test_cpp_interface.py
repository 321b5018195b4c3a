"""The C++ mirror of SMAX::Interface (include/smax_b200.hpp): compiled with
g++ against the C ABI library and run as a program that checks every result
against host loops.  Without a GPU the program checks the clean error path."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "smaxkernels_b200")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("cpp") / "interface_test")
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(REPO, "include"),
           os.path.join(REPO, "tests", "cpp", "interface_test.cpp"), "-L", PKG, "-l:libsmax_b200.so",
           f"-Wl,-rpath,{PKG}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_cpp_interface_without_gpu(program):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present: the GPU test runs the full program")
    r = subprocess.run([program, "--no-gpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASS" in r.stdout


@pytest.mark.gpu
def test_cpp_interface_on_gpu(program):
    r = subprocess.run([program], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("PASS") == 9 and "FAIL" not in r.stdout
