"""The C ABI header is plain C: a minimal C caller (tests/c/minimal_example.c) compiles against it
(C99, all warnings as errors)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_minimal_c_example_compiles(tmp_path):
    src = os.path.join(ROOT, "tests", "c", "minimal_example.c")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        "-c", src, "-o", str(tmp_path / "example.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
