"""GPU parity of the float-center mode against the FP64 oracle.

The reference keeps uint8 centers (kmeans.cu:367); this mode keeps fp32 centers computed in FP64
from exact integer sums, takes distances from the tensor cores with hi + lo bf16 centers and fp32
accumulation, and re-scores in FP64 every descriptor whose margin is within the error bound.  So
the assignments -- and therefore the centers, occurrence counts and word IDs -- must be identical
to the oracle's FP64 evaluation (oracle/rbw_oracle.cpp, orc_build_vocabulary_f32 /
orc_lookup_f32), and centers within 1e-5 relative of its FP64 means."""
import os

import numpy as np
import pytest
import torch

import rapidbow_b200 as rbw
from oracle.pyoracle import INIT_INJECTED, INIT_KMEANSPP, level_beg
from rapidbow_b200.synth import sift_like
from tests.helpers import edge_descriptors, random_tree

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _lookup(voc, desc_np):
    out = voc.lookup(torch.from_numpy(desc_np).cuda())
    torch.cuda.synchronize()
    assert voc.device_errors() == (0, 0)
    return out.cpu().numpy().view(np.uint32)


def _rel(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)))


def test_integer_valued_float_tree_equals_uint8_tree(oracle):
    """fp32 centers holding integers: FP64 distances are exact integers, so the float lookup must
    equal the uint8 lookup of the same tree, duplicate centers (exact ties) included."""
    for B, L, seed in [(16, 3, 1), (10, 4, 2), (3, 6, 3)]:
        centers, masks, weights = random_tree(B, L, seed=seed, dup_rate=0.3)
        v8 = rbw.vocabulary_from_host(B, L, centers, masks, weights)
        vf = rbw.vocabulary_from_host_f32(B, L, centers.astype(np.float32), masks, weights)
        assert vf.float_centers and not v8.float_centers
        desc = edge_descriptors(centers, 20011, seed=seed + 10)
        want = oracle.lookup(centers, B, L, desc, threads=THREADS)
        assert np.array_equal(_lookup(v8, desc), want)
        assert np.array_equal(_lookup(vf, desc), want)
        assert np.array_equal(oracle.lookup_f32(centers.astype(np.float32), B, L, desc, threads=THREADS), want)
        assert vf.refined_lookups() > 0  # exact ties are always re-scored


def test_float_lookup_near_ties_match_fp64_oracle(oracle):
    """Pairs of centers that differ by a fraction of a unit in a few dimensions put many
    descriptors within the error bound; the re-score must settle each of them exactly as FP64."""
    rng = np.random.default_rng(5)
    data = sift_like(40000, seed=5).numpy()
    B, L = 16, 3
    nodes = level_beg(B, L)
    centers = data[rng.integers(0, data.shape[0], nodes * B)].reshape(nodes, B, 128).astype(np.float32)
    centers += rng.uniform(-0.5, 0.5, centers.shape).astype(np.float32)
    for b in range(1, B, 2):  # odd centers: near copies of the even ones
        centers[:, b] = centers[:, b - 1]
        centers[:, b, :4] += rng.uniform(-0.05, 0.05, (nodes, 4)).astype(np.float32)
    masks = np.full(nodes, (1 << B) - 1, np.uint32)
    weights = np.ones((nodes, B), np.float32)
    voc = rbw.vocabulary_from_host_f32(B, L, centers, masks, weights)
    desc = np.concatenate([data, sift_like(60000, seed=6).numpy()])
    voc.refined_lookups()
    got = _lookup(voc, desc)
    refined = voc.refined_lookups()
    want = oracle.lookup_f32(centers, B, L, desc, threads=THREADS)
    assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} of {got.size} differ"
    # every center has a near copy, so nearly every descriptor is re-scored at every level
    assert 0.5 * 3 * desc.shape[0] < refined <= 3 * desc.shape[0]


def test_float_blob_round_trip_and_rounded_tree():
    rng = np.random.default_rng(7)
    B, L = 10, 3
    nodes = level_beg(B, L)
    centers = rng.uniform(0, 255, (nodes, B, 128)).astype(np.float32)
    masks = np.full(nodes, (1 << B) - 1, np.uint32)
    weights = rng.uniform(0.1, 2, (nodes, B)).astype(np.float32)
    voc = rbw.vocabulary_from_host_f32(B, L, centers, masks, weights)
    blob = voc.serialize()
    voc2 = rbw.deserialize_vocabulary(blob)
    assert voc2.float_centers
    assert np.array_equal(voc2.centers_f32(), centers)
    assert voc2.serialize() == blob
    c8, m, w = voc2.tree()
    assert np.array_equal(c8, np.clip(np.rint(centers), 0, 255).astype(np.uint8))
    assert np.array_equal(m, masks) and np.array_equal(w, weights)
    with pytest.raises(rbw.RbwError) as e:
        rbw.deserialize_vocabulary(blob[:-4])
    assert e.value.status == rbw.RBW_ERR_INVALID_BLOB
    with pytest.raises(rbw.RbwError) as e:
        voc.lookup_noalloc(torch.zeros((4, 128), dtype=torch.uint8, device="cuda"),
                           torch.zeros(4, dtype=torch.int32, device="cuda"))
    assert e.value.status == rbw.RBW_ERR_UNSUPPORTED
    with pytest.raises(rbw.RbwError) as e:
        rbw.vocabulary_from_host(B, L, c8, masks, weights).centers_f32()
    assert e.value.status == rbw.RBW_ERR_UNSUPPORTED


def _check_float_build(oracle, desc, B, L, init, seed=0, injected=None, fresh=None):
    dev = torch.from_numpy(desc).cuda()
    voc = rbw.build_vocabulary(dev, B, nb_doc=1000, nb_levels=L, init=init, seed=seed, injected=injected,
                               max_iterations=10, check_interval=4, float_centers=True)
    ref = oracle.build_vocabulary_f32(desc, 1000, B, L, max_iter=10,
                                      init={"kmeans++": INIT_KMEANSPP, "injected": INIT_INJECTED}[init], seed=seed,
                                      injected=injected, threads=THREADS)
    got = voc.centers_f32()
    assert _rel(got, ref["centers"]) <= 1e-5
    assert np.array_equal(got, ref["centers"]), "centers differ from the FP64 oracle"
    c8, masks, weights = voc.tree()
    assert np.array_equal(masks, ref["masks"])
    assert np.array_equal(weights, ref["weights"]), "occurrence counts (assignments) differ"
    st = voc.build_stats()
    assert st["levels"] == L
    for lv in range(L):
        assert abs(st["inertia_first"][lv] - ref["inertia_first"][lv]) <= 1e-9 * ref["inertia_first"][lv]
        assert abs(st["inertia_last"][lv] - ref["inertia_last"][lv]) <= 1e-9 * ref["inertia_last"][lv]
        assert st["inertia_last"][lv] <= st["inertia_first"][lv]
        assert st["refined"][lv] <= st["assignments"][lv]
    assert sum(st["refined"]) > 0
    for x in [desc] + ([fresh] if fresh is not None else []):
        assert np.array_equal(_lookup(voc, x), oracle.lookup_f32(ref["centers"], B, L, x, threads=THREADS))
    return voc, ref, st


def test_float_build_matches_fp64_oracle_b16(oracle):
    desc = sift_like(60000, seed=31).numpy()
    _check_float_build(oracle, desc, 16, 3, "kmeans++", seed=9, fresh=sift_like(20000, seed=32).numpy())


def test_float_build_zipf_1m_b10_l4_injected_init(oracle):
    """The 10M-descriptor, 4,096-component Zipf(1.1) workload's generator at 1M descriptors, a
    10-ary, 4-level tree, injected initial centers (random descriptor rows, some slots invalid)
    and 10 Lloyd iterations."""
    B, L = 10, 4
    n = 1_000_000
    desc = sift_like(n, seed=41, n_components=4096, zipf=1.1, device="cuda").cpu().numpy()
    rng = np.random.default_rng(42)
    nodes = level_beg(B, L)
    injected = rng.integers(0, n, (nodes, B)).astype(np.uint32)
    injected[rng.random(nodes) < 0.05, B - 1] = 0xFFFFFFFF  # an invalid last slot in 5% of the nodes
    fresh = sift_like(200_000, seed=43, n_components=4096, zipf=1.1, device="cuda").cpu().numpy()
    _check_float_build(oracle, desc, B, L, "injected", injected=injected, fresh=fresh)


def test_uint8_build_injected_init_matches_oracle(oracle):
    """The uint8 mode with injected initial centers (RBW_INIT_INJECTED) on the Zipf generator:
    byte-identical to the oracle (IEEE rounding of the quotient, as the oracle divides)."""
    B, L = 10, 4
    n = 300_000
    desc = sift_like(n, seed=51, n_components=4096, zipf=1.1, device="cuda").cpu().numpy()
    rng = np.random.default_rng(52)
    nodes = level_beg(B, L)
    injected = rng.integers(0, n, (nodes, B)).astype(np.uint32)
    injected[rng.random(nodes) < 0.05, B - 1] = 0xFFFFFFFF
    voc = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), B, nb_doc=1000, nb_levels=L, init="injected",
                               injected=injected, max_iterations=10, ieee_division=True)
    ref = oracle.build_vocabulary(desc, 1000, B, L, max_iter=10, init=INIT_INJECTED, injected=injected)
    c, m, w = voc.tree()
    assert np.array_equal(c, ref["centers"])
    assert np.array_equal(m, ref["masks"])
    assert np.array_equal(w, ref["weights"])
    assert np.array_equal(_lookup(voc, desc), oracle.lookup(ref["centers"], B, L, desc, threads=THREADS))
