"""rbw_voc_lookup_noalloc: the lookup for callers that cannot allocate device memory during the
call (latency-bound serving loops, plug-ins inside an application that owns the GPU memory,
fixed memory budgets).  Its working memory is a
fixed array inside the library, shared by all calls on a GPU and kept between calls, so two
calls in a row must each give the same leaf IDs as the allocating entry point.  This file is
collected last so that a run stopping at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

import rapidbow_b200 as rbw
from tests.helpers import edge_descriptors, random_tree

pytestmark = pytest.mark.gpu


def test_noalloc_lookup_matches_allocating_lookup_on_two_calls():
    B, L = 16, 4
    centers, masks, weights = random_tree(B, L, seed=77)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    for n, seed in [(300_001, 1), (123_457, 2)]:  # second call: smaller, different data
        desc = torch.from_numpy(edge_descriptors(centers, n, seed)).cuda()
        want = voc.lookup(desc, algo="tensor_u8")
        got = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        voc.lookup_noalloc(desc, got)
        torch.cuda.synchronize()
        assert voc.device_errors() == (0, 0)
        assert torch.equal(got, want)


def test_noalloc_rejects_calls_beyond_its_fixed_array():
    B, L = 16, 4
    centers, masks, weights = random_tree(B, L, seed=78)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    n = 4_000_000  # needs about 33 MB of working memory
    assert voc.scratch_bytes(n) > 8 << 20
    lib = rbw.load_library()
    rc = lib.rbw_voc_lookup_noalloc(voc.handle, C.c_void_p(16), n, C.c_void_p(16), None)
    assert rc == rbw.RBW_ERR_INVALID_ARG
    assert b"fixed" in lib.rbw_last_error()
