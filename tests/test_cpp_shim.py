"""The C++ face (include/oapb200.hpp): a small C++ program written against
the reference's class and method names (CuProceduresApi, CuHArnoldiCallback,
MatrixInfo, ArnUtils sort orders, testOutcome) is compiled with g++ and run:
argument checks and error conversion on the CPU, the operator surface, QRGR
and dense / callback solves of a planted spectrum on the GPU."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def shim_binary(tmp_path_factory):
    lib = os.path.join(ROOT, "oap_b200", "liboapb200.so")
    if not os.path.exists(lib):
        pytest.skip("liboapb200.so not built")
    out = str(tmp_path_factory.mktemp("shim") / "shim_test")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "shim_test.cpp"),
           "-L", os.path.join(ROOT, "oap_b200"), "-loapb200", "-Wl,-rpath," + os.path.join(ROOT, "oap_b200"),
           "-L", os.path.join(CUDA, "lib64"), "-lcudart_static", "-ldl", "-lrt", "-lpthread", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_cpp_shim_cpu(shim_binary):
    r = subprocess.run([shim_binary, "cpu"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpu: 0 failures" in r.stdout


@pytest.mark.gpu
def test_cpp_shim_gpu(shim_binary):
    r = subprocess.run([shim_binary, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "gpu: 0 failures" in r.stdout
