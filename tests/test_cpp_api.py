"""The rbow:: C++ interface (include/RapidBoW.h) compiles, links against librapidbow_b200.so and,
on a GPU, runs the reference's end-to-end flow (tests/cpp/api_test.cpp)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "rapidbow_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path) -> str:
    exe = str(tmp_path / "api_test")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "api_test.cpp"), "-o", exe, "-L", LIBDIR, "-lrapidbow_b200",
           "-Wl,-rpath," + LIBDIR, "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_interface_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "librapidbow_b200.so")):
        pytest.skip("library not built")
    _build(tmp_path)


@pytest.mark.gpu
def test_cpp_interface_end_to_end(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "api_test: ok" in r.stdout
