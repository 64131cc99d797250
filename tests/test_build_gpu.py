"""GPU hierarchical k-means build (Vocabulary.cpp:32-121, kmeans.cpp) against the oracle and the
reference's own build.

The reference rounds centers with its --use_fast_math division (kmeans.cu:367); the oracle
divides with IEEE division.  Comparisons with the oracle therefore build with
ieee_division=True, and the default (reference) rounding is pinned against the reference's own
build, bit for bit."""
import numpy as np
import pytest
import torch

import rapidbow_b200 as rbw
from oracle.pyoracle import INIT_KMEANSPP, INIT_REFERENCE, parse_reference_blob
from rapidbow_b200.synth import sift_like

pytestmark = pytest.mark.gpu


def _tree_equal(voc, ref):
    c, m, w = voc.tree()
    assert np.array_equal(m, ref["masks"]), "masks differ"
    bad = np.argwhere(c != ref["centers"])
    assert bad.size == 0, f"{len(bad)} center bytes differ, first at {bad[:3].tolist()}"
    assert np.array_equal(w, ref["weights"]), "weights differ"


@pytest.mark.parametrize("B,L,n", [(16, 2, 3000), (16, 3, 20000), (10, 3, 8000), (4, 4, 1500)])
def test_build_reference_init_matches_oracle(oracle, B, L, n):
    desc = sift_like(n, seed=B + L).numpy()
    voc = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), B, nb_doc=77, nb_levels=L, ieee_division=True)
    ref = oracle.build_vocabulary(desc, 77, B, L, max_iter=1000, init=INIT_REFERENCE)
    _tree_equal(voc, ref)


@pytest.mark.parametrize("B,L,n,iters", [(16, 3, 20000, 10), (10, 3, 10000, 10), (16, 2, 5000, 1000)])
def test_build_kmeanspp_matches_oracle(oracle, B, L, n, iters):
    desc = sift_like(n, seed=100 + B).numpy()
    voc = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), B, nb_doc=50, nb_levels=L, init="kmeans++", seed=1234,
                               max_iterations=iters, ieee_division=True)
    ref = oracle.build_vocabulary(desc, 50, B, L, max_iter=iters, init=INIT_KMEANSPP, seed=1234)
    _tree_equal(voc, ref)


@pytest.mark.parametrize("n_distinct,n", [(6, 3000), (40, 600), (300, 5000)])
def test_build_kmeanspp_duplicates_match_oracle(oracle, n_distinct, n):
    """Few distinct rows: the D^2 weights reach zero before B picks (fewer valid centers, empty
    children at the next level) and the sampled candidates repeat."""
    base = sift_like(n_distinct, seed=321 + n_distinct).numpy()
    desc = np.ascontiguousarray(base[np.random.default_rng(n).integers(0, n_distinct, n)])
    voc = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), 16, nb_doc=20, nb_levels=2, init="kmeans++", seed=99,
                               max_iterations=10, ieee_division=True)
    ref = oracle.build_vocabulary(desc, 20, 16, 2, max_iter=10, init=INIT_KMEANSPP, seed=99)
    _tree_equal(voc, ref)


def test_build_matches_reference_build(reference):
    """Bit-identical blob with the reference's own buildVocabulary (same default-seeded RNG)."""
    desc = sift_like(30000, seed=77).numpy()
    blob_ref = reference.build_vocabulary(desc, nb_doc=123, L=3)
    voc = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), 16, nb_doc=123, nb_levels=3)
    blob = voc.serialize()
    if blob != blob_ref:
        L, c, m, w = parse_reference_blob(blob_ref)
        _tree_equal(voc, dict(centers=c, masks=m, weights=w))
    assert blob == blob_ref


def test_build_matches_reference_build_ten_iterations(reference):
    desc = sift_like(20000, seed=78).numpy()
    blob_ref = reference.build_vocabulary(desc, nb_doc=10, L=3, max_iter=10, check_interval=4)
    voc = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), 16, nb_doc=10, nb_levels=3, max_iterations=10)
    assert voc.serialize() == blob_ref


def test_ref_check_full_every_descriptor_is_its_own_leaf():
    """tests/VocTests.cpp:86-132: 32 random descriptors, 3 levels -> inertia 0."""
    rng = np.random.default_rng(0)
    desc = rng.integers(0, 256, size=(32, 128), dtype=np.uint8)
    d = torch.from_numpy(desc).cuda()
    voc = rbw.build_vocabulary(d, 16, nb_doc=4, nb_levels=3)
    leaf = voc.lookup(d).cpu().numpy().view(np.uint32)
    c, _, _ = voc.tree()
    leaves = c[1 + 16:].reshape(-1, 128)
    assert np.all(leaves[leaf] == desc)


def test_ref_check_2d_rms_below_ten():
    """tests/VocTests.cpp:38-84: only bytes 126-127 random, 2 levels -> RMS to leaf <= 10."""
    rng = np.random.default_rng(0)
    desc = np.zeros((4096, 128), np.uint8)
    desc[:, 126:128] = rng.integers(0, 256, size=(4096, 2), dtype=np.uint8)
    d = torch.from_numpy(desc).cuda()
    voc = rbw.build_vocabulary(d, 16, nb_doc=16, nb_levels=2)
    leaf = voc.lookup(d).cpu().numpy().view(np.uint32)
    c, _, _ = voc.tree()
    cent = c[1:].reshape(-1, 128)[leaf].astype(np.int64)
    rms = np.sqrt(((desc.astype(np.int64) - cent) ** 2).sum(1).mean())
    assert rms <= 10


def test_build_rejects_bad_input():
    d = torch.zeros((10, 128), dtype=torch.uint8, device="cuda")
    with pytest.raises(rbw.RbwError) as e:
        rbw.build_vocabulary(d, 16, nb_doc=1, nb_levels=2)
    assert "Insufficient descriptors" in str(e.value)
    d = torch.zeros((100, 128), dtype=torch.uint8, device="cuda")
    with pytest.raises(rbw.RbwError):
        rbw.build_vocabulary(d, 16, nb_doc=0, nb_levels=2)
    with pytest.raises(rbw.RbwError) as e:
        rbw.build_vocabulary(d, 17, nb_doc=1, nb_levels=2)
    assert e.value.status == rbw.RBW_ERR_UNSUPPORTED
