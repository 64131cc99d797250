"""Pins the oracle (CPU restatement, oracle/) to the reference itself.

Two sources: the golden fixtures in tests/golden/ (outputs of the reference library, compiled
from its sources, made by tests/golden/make_golden.py on a GPU machine) and, where the
reference library is built here (oracle/_ref), its CPU DataBase run live.  CPU only.
"""
import os

import numpy as np
import pytest

from oracle.pyoracle import parse_reference_blob
from tests.helpers import random_tree

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.fail(f"golden fixture {name} is missing (tests/golden/make_golden.py makes it)")
    return np.load(path)


def test_lookup_matches_reference_build_and_lookup(oracle):
    g = _load("voc_b16_l2.npz")
    L, centers, masks, weights = parse_reference_blob(g["blob"].tobytes())
    assert L == 2 and np.all(masks == 0xFFFF)
    assert np.array_equal(oracle.lookup(centers, 16, 2, g["queries"]), g["leaves"])


def test_lookup_matches_reference_random_tree(oracle):
    g = _load("lookup_b16_l3.npz")
    centers, _, _ = random_tree(16, 3, int(g["tree_seed"]))
    assert np.array_equal(oracle.lookup(centers, 16, 3, g["queries"]), g["leaves"])


def test_kmeans_assign_matches_reference_kernel(oracle):
    g = _load("kmeans_task.npz")
    for t in range(4):
        desc = g[f"t{t}_desc"]
        members = np.arange(desc.shape[0], dtype=np.uint32)
        assign, counts, sums, changed = oracle.kmeans_assign(desc, members, g[f"t{t}_centers"], 16, g[f"t{t}_prev"])
        assert np.array_equal(assign, g[f"t{t}_assign"])
        assert np.array_equal(counts, g[f"t{t}_counts"])
        assert np.array_equal(sums, g[f"t{t}_sums"].astype(np.uint64))
        assert changed == int(g[f"t{t}_changed"])


def test_kmeans_update_matches_reference_up_to_half_ties(oracle):
    """The reference rounds float(sum) / count computed with --use_fast_math; the oracle divides
    exactly.  They agree wherever the quotient is not within rounding of a .5 tie."""
    g = _load("kmeans_task.npz")
    for t in range(4):
        counts = g[f"t{t}_counts"]
        sums = g[f"t{t}_sums"].astype(np.uint64)
        mine = oracle.kmeans_update(counts, sums, g[f"t{t}_centers"])
        want = g[f"t{t}_updated"]
        n = counts[:, None].astype(np.float64)
        q = np.where(n > 0, sums.astype(np.float64) / np.maximum(n, 1), 0)
        tie = np.abs(q - np.floor(q) - 0.5) < 1e-6
        ok = (mine == want) | (tie & (np.abs(mine.astype(int) - want.astype(int)) <= 1))
        assert ok.all()


def _db_fixture(oracle):
    g = _load("db_b16_l3.npz")
    odb = oracle.db(16, 3, g["weights"])
    offs = g["doc_offsets"]
    for i, d in enumerate(g["doc_ids"]):
        odb.add(int(d), g["doc_leaves"][int(offs[i]): int(offs[i + 1])])
    qoff = g["query_offsets"]
    queries = [g["query_leaves"][int(qoff[j]): int(qoff[j + 1])] for j in range(qoff.size - 1)]
    return g, odb, queries


def _same_ranking(all_docs, all_scores, want):
    """The oracle's first len(want) documents equal `want`, or differ only among documents of
    equal oracle score (the reference's std::sort leaves their order open).  all_docs /
    all_scores: every touched document, sorted by (score, id)."""
    n = want.size
    if np.array_equal(all_docs[:n], want):
        return True
    s = dict(zip(all_docs.tolist(), all_scores.tolist()))
    if not set(want.tolist()) <= set(s):
        return False
    b = np.array([s[int(x)] for x in want])
    return bool(np.all(all_scores[:n] == b))


@pytest.mark.parametrize("k", [10, 50])
def test_database_matches_reference_golden(oracle, k):
    g, odb, queries = _db_fixture(oracle)
    for j, q in enumerate(queries):
        docs, scores = odb.query(q, k, mode=0)
        n = int(g[f"k{k}_counts"][j])
        assert min(k, docs.size) == n
        want = g[f"k{k}_results"][j, :n]
        # rank through the oracle's full list so that ties at the cut are handled
        assert _same_ranking(docs, scores, want), f"query {j}"


def test_database_matches_live_reference(oracle, reference):
    """The reference's CPU DataBase against the oracle on fresh random databases (B=16, L=2..4)."""
    rng = np.random.default_rng(3)
    for L, n_docs in ((2, 60), (3, 200), (4, 150)):
        _, _, w = random_tree(16, L, 10 + L)
        n_leaves = 16 ** L
        rdb, odb = reference.db(L, w), oracle.db(16, L, w)
        docs = [rng.integers(0, n_leaves, size=int(rng.integers(1, 300)), dtype=np.uint32) for _ in range(n_docs)]
        for i, d in enumerate(docs):
            rdb.add(i * 5 + 1, d)
            odb.add(i * 5 + 1, d)
            assert np.float32(odb.doc_rcp(i * 5 + 1)) > 0
        for j in range(15):
            q = np.concatenate([docs[j][: docs[j].size // 2], rng.integers(0, n_leaves, size=30, dtype=np.uint32)])
            for k in (3, 40, 1000):
                want = rdb.query(q.astype(np.uint32), k)
                got, scores = odb.query(q.astype(np.uint32), k, mode=0)
                assert want.size == min(k, got.size)
                assert _same_ranking(got, scores, want)
        # postings: sorted ids with duplicates
        leaf = int(docs[0][0])
        assert np.all(np.diff(odb.postings(leaf).astype(np.int64)) >= 0)
