"""The C ABI header is plain C, and the minimal C example in INTEGRATION.md compiles against it
(C99, all warnings as errors)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _example():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"### Minimal C use\s*```c\n(.*?)```", text, re.S)
    assert m, "INTEGRATION.md has no minimal C example"
    lines = m.group(1).splitlines()
    includes = [l for l in lines if l.startswith("#include")]
    body = [l for l in lines if not l.startswith("#include")]
    return includes, body


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_minimal_c_example_compiles(tmp_path):
    includes, body = _example()
    src = "\n".join(["#include <stdio.h>", *includes,
                     "int example(const void* dev_desc, uint32_t n_train, uint32_t n_docs,",
                     "            const void* dev_query_desc, uint32_t n_query, uint32_t* dev_leaf_ids, void* stream)",
                     "{", *["    " + l for l in body], "    return 0;", "}", ""])
    path = tmp_path / "example.c"
    path.write_text(src)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        "-c", str(path), "-o", str(tmp_path / "example.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr + "\n" + src
