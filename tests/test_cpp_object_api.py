"""The C++ object API (include/b3gpu.hpp) driven from a C++ host program,
tests/cpp/object_api_test.cpp, compiled against the built library."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "object_api_test.cpp")
LIBDIR = os.path.join(ROOT, "experiments_b200", "lib")
OUT = os.path.join(ROOT, "experiments_b200", "_build", "object_api_test")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def program():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"), SRC,
           "-L", LIBDIR, "-lb3gpu", "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{LIBDIR}",
           f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}", "-o", OUT]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return OUT


def test_object_api_host(program):
    bullet = os.path.join(ROOT, "tests", "golden", "pile.bullet")  # a .bullet scene of 41 bodies
    r = subprocess.run([program, "host", bullet], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_object_api_gpu(program):
    r = subprocess.run([program, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
