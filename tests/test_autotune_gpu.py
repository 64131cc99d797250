"""The autotuner on the GPU: every candidate of every tunable parameter gives the same results
(the parameters change launch shapes only), and tuning on a real workload records and applies
the fastest candidate."""
import numpy as np
import pytest
import torch

import rapidbow_b200 as rbw
from rapidbow_b200 import autotune as at
from rapidbow_b200.synth import sift_like
from tests.helpers import edge_descriptors, random_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _clean():
    at.clear()
    yield
    at.clear()


def test_scatter_rows_candidates_are_exact(oracle):
    """B=10, L=6: the regroup after the second pass has 10,000 bins, which takes the scatter
    whose rows per thread are tuned."""
    B, L = 10, 6
    centers, masks, weights = random_tree(B, L, seed=91)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    n = 300_007
    host = edge_descriptors(centers, n, seed=92)
    desc = torch.from_numpy(host).cuda()
    want = oracle.lookup(centers, B, L, host, threads=8)
    for rows in at.CANDIDATES["scatter_rows"]:
        at.set_value("scatter_rows", B, L, at.bucket(n), rows)
        got = voc.lookup(desc, algo="tensor_u8")
        torch.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy().view(np.uint32), want), rows
    for sched in at.CANDIDATES["lookup_schedule"]:
        at.set_value("lookup_schedule", B, L, at.bucket(n), sched)
        got = voc.lookup(desc)  # algo "auto" runs the tuned schedule
        torch.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy().view(np.uint32), want), sched


@pytest.mark.parametrize("float_centers", [False, True])
def test_assign_grid_candidates_give_identical_builds(float_centers):
    B, L = 10, 3
    desc = sift_like(100_000, seed=93, n_components=4096, zipf=1.1, device="cuda")
    param = "assign_f32_ctas_per_sm" if float_centers else "assign_ctas_per_sm"
    trees = []
    for v in at.CANDIDATES[param]:
        at.set_value(param, B, 0, at.bucket(desc.shape[0]), v)
        voc = rbw.build_vocabulary(desc, B, nb_doc=100, nb_levels=L, init="kmeans++", seed=3, max_iterations=6,
                                   float_centers=float_centers)
        trees.append((voc.centers_f32() if float_centers else voc.tree()[0], voc.tree()[2]))
    for c, w in trees[1:]:
        assert np.array_equal(c, trees[0][0]) and np.array_equal(w, trees[0][1])


def test_tensor_core_sums_give_the_oracle_build(oracle):
    """Center sums from the second MMA per tile (assign_sums = 2, rows gathered one tile ahead)
    equal the shared-atomic sums: the IEEE-rounding build equals the oracle's byte for byte, on a
    one-node level of 150,000 members (a node spread over many CTAs) and on small nodes."""
    from oracle.pyoracle import INIT_KMEANSPP

    desc_t = sift_like(150_000, seed=96, n_components=4096, zipf=1.1, device="cuda")
    desc = desc_t.cpu().numpy()
    B, L = 10, 3
    at.set_value("assign_sums", B, 0, at.bucket(desc.shape[0]), 2)
    for ctas in (2, 4):
        at.set_value("assign_ctas_per_sm", B, 0, at.bucket(desc.shape[0]), ctas)
        voc = rbw.build_vocabulary(desc_t, B, nb_doc=100, nb_levels=L, init="kmeans++", seed=3, max_iterations=10,
                                   ieee_division=True)
        ref = oracle.build_vocabulary(desc, 100, B, L, max_iter=10, init=INIT_KMEANSPP, seed=3)
        c, m, w = voc.tree()
        assert np.array_equal(c, ref["centers"]) and np.array_equal(m, ref["masks"]), ctas
        assert np.array_equal(w, ref["weights"]), ctas


@pytest.mark.parametrize("B,L,n,nb_doc", [(16, 3, 30000, 123), (10, 4, 60000, 50)])
def test_tensor_core_sums_give_the_reference_build(reference, B, L, n, nb_doc):
    """The tensor-core sums with the reference's fast-math center division: the B = 16 blob
    equals the reference's own build, and with B = 10 (no reference build) the tree equals the
    build with shared-atomic sums."""
    desc_t = sift_like(n, seed=77 + B, device="cuda")
    desc = desc_t.cpu().numpy()
    at.set_value("assign_sums", B, 0, at.bucket(n), 2)
    voc = rbw.build_vocabulary(desc_t, B, nb_doc=nb_doc, nb_levels=L, max_iterations=1000)
    if B == 16:
        assert voc.serialize() == reference.build_vocabulary(desc, nb_doc=nb_doc, L=L)
    at.set_value("assign_sums", B, 0, at.bucket(n), 1)
    base = rbw.build_vocabulary(desc_t, B, nb_doc=nb_doc, nb_levels=L, max_iterations=1000)
    for a, b in zip(voc.tree(), base.tree()):
        assert np.array_equal(a, b)


def test_tuning_records_the_fastest_and_applies_it(tmp_path):
    t = at.Autotuner.for_current_device(str(tmp_path / "tune.json"))
    B, L = 16, 4
    train = sift_like(200_000, seed=94, device="cuda")
    e = t.tune_build(train, B, 3, nb_doc=100, init="kmeans++", seed=1, max_iterations=4)
    assert e["value"] in at.CANDIDATES["assign_ctas_per_sm"] and e["ms"] > 0
    assert e["ms"] == min(e["candidates"].values())
    voc = rbw.build_vocabulary(train, B, nb_doc=100, nb_levels=L, init="kmeans++", seed=1, max_iterations=4)
    desc = sift_like(1_000_000, seed=95, device="cuda")
    e2 = t.tune_lookup(voc, desc)
    assert e2["value"] in at.CANDIDATES["lookup_schedule"]
    assert at.get_value("lookup_schedule", B, L, desc.shape[0]) == e2["value"]
    t.save()
    at.clear()
    t2 = at.Autotuner.for_current_device(t.path)
    assert t2.load() and t2.apply() == 3  # assign sums, assign CTAs per SM, lookup schedule
    assert at.get_value("lookup_schedule", B, L, desc.shape[0]) == e2["value"]
