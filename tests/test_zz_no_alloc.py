"""rbw_voc_lookup_noalloc: the lookup for callers that cannot allocate device memory during the
call (latency-bound serving loops, plug-ins inside an application that owns the GPU memory,
fixed memory budgets).  Its working memory is a fixed 8 MiB array inside the library, shared by
all calls on a GPU and kept between calls, so two calls in a row must each give the same leaf
IDs as the allocating entry point and as the oracle, including the largest call that fits the
array (where the tile list ends at the array's last bytes).  This file is collected last so
that a run stopping at the first failure has already run every other test."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

import rapidbow_b200 as rbw
from tests.helpers import edge_descriptors, random_tree

pytestmark = pytest.mark.gpu

ARRAY_BYTES = 8 << 20


def _largest_n(voc) -> int:
    """Largest descriptor count whose lookup working memory fits the fixed array."""
    lo, hi = 1, 1 << 24
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if voc.scratch_bytes(mid) <= ARRAY_BYTES:
            lo = mid
        else:
            hi = mid - 1
    return lo


def test_noalloc_lookup_matches_oracle_and_allocating_lookup_on_two_calls(oracle):
    B, L = 16, 4
    centers, masks, weights = random_tree(B, L, seed=77)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    n_max = _largest_n(voc)
    assert 1_000_000 < n_max < 1_100_000
    threads = os.cpu_count() or 1
    # second call smaller, different data: nothing of the first call's contents may leak into it
    for n, seed in [(n_max, 1), (123_457, 2)]:
        host = edge_descriptors(centers, n, seed)
        desc = torch.from_numpy(host).cuda()
        want = voc.lookup(desc, algo="tensor_u8")
        got = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        voc.lookup_noalloc(desc, got)
        torch.cuda.synchronize()
        assert voc.device_errors() == (0, 0)
        assert torch.equal(got, want)
        assert np.array_equal(got.cpu().numpy().view(np.uint32), oracle.lookup(centers, B, L, host, threads=threads))


def test_noalloc_rejects_calls_beyond_its_fixed_array():
    B, L = 16, 4
    centers, masks, weights = random_tree(B, L, seed=78)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    lib = rbw.load_library()
    for n in (_largest_n(voc) + 1, 4_000_000):
        assert voc.scratch_bytes(n) > ARRAY_BYTES
        rc = lib.rbw_voc_lookup_noalloc(voc.handle, C.c_void_p(16), n, C.c_void_p(16), None)
        assert rc == rbw.RBW_ERR_INVALID_ARG
        assert b"fixed" in lib.rbw_last_error()
