"""GPU parity of the tree descent (vocTreeLookUp.cu:82-155 semantics): word IDs must be
bit-identical to the oracle and to the reference's own kernel, for every algorithm."""
import numpy as np
import pytest
import torch

import rapidbow_b200 as rbw
from tests.helpers import edge_descriptors, random_tree

pytestmark = pytest.mark.gpu

ALGOS = ["tensor_u8", "simt_f32", "tensor_u8_warpnode", "tensor_u8_ring"]


def _lookup(voc, desc_np, algo):
    d = torch.from_numpy(desc_np).cuda()
    out = voc.lookup(d, algo=algo)
    torch.cuda.synchronize()
    assert voc.device_errors() == (0, 0)
    return out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("B,L", [(16, 1), (16, 2), (16, 3), (16, 4), (10, 3), (10, 4), (2, 7), (3, 5), (16, 5)])
@pytest.mark.parametrize("algo", ALGOS)
def test_lookup_matches_oracle(oracle, B, L, algo):
    centers, masks, weights = random_tree(B, L, seed=B * 100 + L)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    for n, seed in [(1, 1), (17, 2), (129, 3), (4099, 4)]:
        desc = edge_descriptors(centers, n, seed)
        got = _lookup(voc, desc, algo)
        want = oracle.lookup(centers, B, L, desc)
        assert np.array_equal(got, want), f"n={n}: {np.count_nonzero(got != want)} mismatches"


@pytest.mark.parametrize("n", [0, 1, 15, 16, 127, 128, 129, 255, 256, 257, 100003, 2000003])
def test_lookup_sizes_tensor_vs_simt_vs_oracle(oracle, n):
    B, L = 16, 4
    centers, masks, weights = random_tree(B, L, seed=7)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    desc = edge_descriptors(centers, n, seed=n)
    a = _lookup(voc, desc, "tensor_u8")
    b = _lookup(voc, desc, "simt_f32")
    assert np.array_equal(a, b)
    assert np.array_equal(_lookup(voc, desc, "tensor_u8_warpnode"), b)
    assert np.array_equal(_lookup(voc, desc, "tensor_u8_ring"), b)
    assert np.array_equal(a, oracle.lookup(centers, B, L, desc, threads=8))


def test_lookup_ties_all_equal_descriptors_and_extremes(oracle):
    B, L = 16, 3
    centers, masks, weights = random_tree(B, L, seed=11, dup_rate=0.5)
    centers[0, :] = centers[0, 5]          # root: every center identical -> branch 0 always
    centers[1, 3] = 0
    centers[1, 4] = 255
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    desc = np.concatenate([np.zeros((300, 128), np.uint8), np.full((300, 128), 255, np.uint8),
                           np.tile(centers[1, 7], (300, 1))])
    for algo in ALGOS:
        got = _lookup(voc, desc, algo)
        assert np.array_equal(got, oracle.lookup(centers, B, L, desc))
        assert np.all(got // 256 == 0)  # tie at the root resolves to branch 0


def test_lookup_sift_like_tree(oracle):
    from rapidbow_b200.synth import sift_like

    data = sift_like(20000, seed=5).numpy()
    B, L = 16, 4
    centers, masks, weights = random_tree(B, L, seed=3, data=data)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    desc = sift_like(50000, seed=6).numpy()
    want = oracle.lookup(centers, B, L, desc, threads=8)
    for algo in ALGOS:
        assert np.array_equal(_lookup(voc, desc, algo), want)


def test_lookup_matches_reference_kernel(reference):
    """The reference's own kernel (built for sm_100a in oracle/_ref) on the same blob."""
    from rapidbow_b200.synth import sift_like

    data = sift_like(20000, seed=8).numpy()
    B, L = 16, 4
    centers, masks, weights = random_tree(B, L, seed=9, data=data)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    blob = voc.serialize()
    desc = np.concatenate([sift_like(30000, seed=10).numpy(), edge_descriptors(centers, 3000, 12)])
    want = reference.lookup(blob, desc)
    for algo in ALGOS:
        assert np.array_equal(_lookup(voc, desc, algo), want)


def test_lookup_host_pipeline_matches_device_path(oracle):
    B, L = 16, 4
    centers, masks, weights = random_tree(B, L, seed=21)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    desc = edge_descriptors(centers, (1 << 20) + 12345, seed=22)
    got = voc.lookup_host(desc)
    assert np.array_equal(got, oracle.lookup(centers, B, L, desc, threads=8))


def test_blob_round_trip_is_byte_exact():
    B, L = 16, 3
    centers, masks, weights = random_tree(B, L, seed=31)
    masks[5] = 0x00FF
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    blob = voc.serialize()
    assert len(blob) == 4 + (1 + 16 + 256) * (2048 + 2 + 64)
    voc2 = rbw.deserialize_vocabulary(blob)
    assert voc2.serialize() == blob
    c, m, w = voc2.tree()
    assert np.array_equal(c, centers) and np.array_equal(m, masks) and np.array_equal(w, weights)
    with pytest.raises(rbw.RbwError) as e:
        rbw.deserialize_vocabulary(blob[:-1])
    assert e.value.status == rbw.RBW_ERR_INVALID_BLOB


def test_blob_extension_for_other_branch_factors():
    B, L = 10, 3
    centers, masks, weights = random_tree(B, L, seed=41)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    voc2 = rbw.deserialize_vocabulary(voc.serialize())
    assert voc2.branch_factor == 10 and voc2.nb_levels == 3
    c, m, w = voc2.tree()
    assert np.array_equal(c, centers) and np.array_equal(w, weights)


def test_lookup_repeated_large_batches_are_exact():
    """Many centre groups per CTA in the gathered pass and a producer that runs ahead of the
    MMA: the double-buffered centre blocks and the row-index ring are reused as fast as the
    hardware allows.  Every repetition must equal the FP32 kernel exactly."""
    from rapidbow_b200.synth import sift_like

    train = sift_like(500_000, seed=21, device="cuda")
    voc = rbw.build_vocabulary(train, 16, nb_doc=1000, nb_levels=4, init="kmeans++", seed=5, max_iterations=5)
    desc = sift_like(8_000_000, seed=22, device="cuda")
    want = voc.lookup(desc, algo="simt_f32")
    for algo in ("tensor_u8", "tensor_u8_warpnode", "tensor_u8_ring"):
        for _ in range(4):
            got = voc.lookup(desc, algo=algo)
            torch.cuda.synchronize()
            assert voc.device_errors() == (0, 0)
            assert int((got != want).sum()) == 0, algo
