"""CPU checks of the drop-in boundary: the C-ABI library loads and exports every declared symbol."""
import ctypes as C
import os
import re

import pytest

import rapidbow_b200 as rbw

HEADERS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_symbols():
    names = set()
    for f in os.listdir(HEADERS):
        if f.endswith(".h"):
            text = open(os.path.join(HEADERS, f)).read()
            names |= set(re.findall(r"RBW_API\s+[\w\s\*]+?\b(rbw_\w+)\s*\(", text))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    lib = rbw.load_library()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if getattr(lib, n, None) is None]
    assert not missing, missing


def test_version_and_defaults():
    lib = rbw.load_library()
    assert b"sm_100a" in lib.rbw_version()
    o = rbw.BuildOptions()
    lib.rbw_build_options_default(C.byref(o))
    assert (o.max_iterations, o.check_interval, o.init_mode) == (1000, 4, 0)


def test_null_handles_are_rejected_without_touching_the_gpu():
    lib = rbw.load_library()
    rc = lib.rbw_voc_info(None, None, None, None, None)
    assert rc == rbw.RBW_ERR_INVALID_ARG
    assert b"null" in lib.rbw_last_error()
    rc = lib.rbw_voc_deserialize(None, 0, C.byref(C.c_void_p()))
    assert rc == rbw.RBW_ERR_INVALID_BLOB


def test_unsupported_attributes_are_rejected():
    lib = rbw.load_library()
    h = C.c_void_p()
    rc = lib.rbw_voc_build(rbw.DescAttr(rbw.DATA_BINARY, rbw.DIST_HAMMING, 256), 16, None, 100, 1, 2, None, None,
                           C.byref(h))
    assert rc == rbw.RBW_ERR_UNSUPPORTED
    assert b"quantized SIFT" in lib.rbw_last_error()
