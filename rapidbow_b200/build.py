"""Build recipe for librapidbow_b200.so (sm_100a only; cross-compiles without a GPU).

Every CUDA / C++ source under csrc/ is compiled with nvcc for ``-gencode
arch=compute_100a,code=sm_100a`` and linked, with the static CUDA runtime, into
``rapidbow_b200/lib/librapidbow_b200.so`` (in-tree, so it travels with the repository).
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "lib", "obj")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(LIBDIR, "librapidbow_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]
# Per-file extra flags: the center update must divide exactly like the reference's
# --use_fast_math kernels.
EXTRA = {"kmeans_update.cu": ["--use_fast_math"]}
SOURCES = ["lookup.cu", "kmeans.cu", "kmeans_update.cu", "kmeans_f32.cu", "vocabulary.cu", "database.cu", "capi.cpp", "facade.cpp",
           "timing.cpp", "noalloc.cu", "server.cpp", "tuning.cpp", "kmeans_shard.cu"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _headers_digest() -> str:
    h = hashlib.sha1()
    for d in (CSRC, INCLUDE):
        for root, _, files in os.walk(d):
            for f in sorted(files):
                if f.endswith((".h", ".cuh", ".hpp")):
                    with open(os.path.join(root, f), "rb") as fh:
                        h.update(fh.read())
    return h.hexdigest()


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    hdr = _headers_digest()

    def compile_one(src: str) -> str:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJDIR, src + ".o")
        stamp = obj + ".stamp"
        with open(path, "rb") as fh:
            key = hashlib.sha1(fh.read() + hdr.encode() + " ".join(EXTRA.get(src, [])).encode()).hexdigest()
        if not force and os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == key:
            return obj
        lang = ["-x", "cu"] if src.endswith(".cu") else []
        cmd = [nvcc, *ARCH, *COMMON, *EXTRA.get(src, []), *lang, "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
        with open(stamp, "w") as fh:
            fh.write(key)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, srcs))
    cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    build_cli(nvcc, verbose)
    return LIB


MAKEVOC = os.path.join(LIBDIR, "makevoc")


def build_cli(nvcc: str, verbose: bool = False) -> str:
    """The makevoc command-line tool (csrc/makevoc.cpp), linked against the library."""
    src = os.path.join(CSRC, "makevoc.cpp")
    cmd = [nvcc, "-O2", "-std=c++17", "-I", INCLUDE, "-x", "cu", src, "-o", MAKEVOC, "-L", LIBDIR, "-lrapidbow_b200",
           "-Xlinker", "-rpath,$ORIGIN", *ARCH]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"makevoc build failed:\n{r.stderr}")
    return MAKEVOC


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
