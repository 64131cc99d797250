"""makevoc, the command-line vocabulary builder (the reference's main.cpp:27-47)."""
import os
import subprocess

import numpy as np
import pytest

MAKEVOC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rapidbow_b200", "lib", "makevoc")


def _need_tool():
    if not os.path.exists(MAKEVOC):
        pytest.skip("makevoc was not built")


def test_usage_and_bad_input(tmp_path):
    _need_tool()
    r = subprocess.run([MAKEVOC], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    r = subprocess.run([MAKEVOC, "--levels", "x", "a", "b"], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"\x00" * 100)  # not a multiple of 128 bytes
    r = subprocess.run([MAKEVOC, str(bad), str(tmp_path / "v.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "128-byte" in r.stderr


@pytest.mark.gpu
def test_blob_equals_library_build(tmp_path):
    import torch

    import rapidbow_b200 as rbw
    from rapidbow_b200.synth import sift_like

    _need_tool()
    desc = sift_like(6000, seed=17).numpy()
    src = tmp_path / "desc.bin"
    src.write_bytes(desc.tobytes())
    out = tmp_path / "voc.bin"
    r = subprocess.run([MAKEVOC, "--docs", "40", "--levels", "2", str(src), str(out)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    voc = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), 16, nb_doc=40, nb_levels=2)
    assert out.read_bytes() == voc.serialize()
    r = subprocess.run([MAKEVOC, "--docs", "40", "--levels", "3", "--branch", "10", "--init", "kmeans++", "--seed", "5",
                        "--iterations", "10", str(src), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    voc2 = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), 10, nb_doc=40, nb_levels=3, init="kmeans++", seed=5,
                                max_iterations=10)
    assert out.read_bytes() == voc2.serialize()
    assert rbw.deserialize_vocabulary(out.read_bytes()).branch_factor == 10
