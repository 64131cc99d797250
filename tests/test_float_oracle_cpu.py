"""CPU checks of the oracle's float-center restatement (the FP64 checker of the float mode)."""
import numpy as np

from oracle.pyoracle import INIT_INJECTED, INIT_KMEANSPP, level_beg
from rapidbow_b200.synth import sift_like


def test_dist64_order_is_a_correct_fp64_sum(oracle):
    rng = np.random.default_rng(1)
    for _ in range(200):
        x = rng.integers(0, 256, 128, dtype=np.uint8)
        c = rng.uniform(0, 255, 128).astype(np.float32)
        exact = float(np.sum((x.astype(np.float64) - c.astype(np.float64)) ** 2))
        assert abs(oracle.dist64(x, c) - exact) <= 1e-12 * exact


def test_dist64_of_integer_centers_is_exact(oracle):
    rng = np.random.default_rng(2)
    x = rng.integers(0, 256, 128, dtype=np.uint8)
    c = rng.integers(0, 256, 128).astype(np.float32)
    assert oracle.dist64(x, c) == float(np.sum((x.astype(np.int64) - c.astype(np.int64)) ** 2))


def test_float_lookup_equals_uint8_lookup_on_integer_trees(oracle):
    from tests.helpers import edge_descriptors, random_tree

    B, L = 16, 3
    centers, _, _ = random_tree(B, L, seed=3, dup_rate=0.3)
    desc = edge_descriptors(centers, 5000, seed=4)
    assert np.array_equal(oracle.lookup_f32(centers.astype(np.float32), B, L, desc, threads=4),
                          oracle.lookup(centers, B, L, desc))


def test_float_build_properties(oracle):
    desc = sift_like(20000, seed=5, n_components=4096, zipf=1.1).numpy()
    B, L = 10, 3
    r1 = oracle.build_vocabulary_f32(desc, 100, B, L, max_iter=10, init=INIT_KMEANSPP, seed=3, threads=1)
    r4 = oracle.build_vocabulary_f32(desc, 100, B, L, max_iter=10, init=INIT_KMEANSPP, seed=3, threads=4)
    for k in ("centers", "masks", "weights", "occ", "iters", "inertia_first", "inertia_last"):
        assert np.array_equal(r1[k], r4[k]), k  # thread count does not change any result
    assert np.all(r1["inertia_last"] <= r1["inertia_first"])
    # every level partitions all descriptors
    for lv in range(L):
        lb, le = level_beg(B, lv), level_beg(B, lv + 1)
        assert int(r1["occ"][lb:le].sum()) == desc.shape[0]
    # fp32 centers are FP64 means of integer rows: within [0, 255]
    assert float(r1["centers"].min()) >= 0.0 and float(r1["centers"].max()) <= 255.0


def test_float_build_init_matches_uint8_init(oracle):
    """Both modes start from the same descriptor rows (injected init, invalid slots = 255)."""
    desc = sift_like(5000, seed=6).numpy()
    B, L = 16, 1
    inj = np.arange(B, dtype=np.uint32).reshape(1, B) * 7
    inj[0, -1] = 0xFFFFFFFF
    rf = oracle.build_vocabulary_f32(desc, 10, B, L, max_iter=1, init=INIT_INJECTED, injected=inj)
    r8 = oracle.build_vocabulary(desc, 10, B, L, max_iter=1, init=INIT_INJECTED, injected=inj)
    assert np.array_equal(rf["masks"], r8["masks"])
    # one Lloyd step against integer centers: the same assignment, so the same counts
    assert np.array_equal(rf["occ"], r8["occ"])
