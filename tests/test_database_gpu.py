"""Parity of the device-resident inverted file (DataBase.cpp:39-197) against the oracle (reference
arithmetic and FP64) and against the reference's own DataBase (oracle/_ref), through the C ABI.

Tolerances: postings, document norms and result ids are exact.  Scores: the reference sums
float terms in double in a fixed order, the kernels sum the same float terms exactly in 64-bit
fixed point, so a score can differ from the reference-arithmetic oracle by one float ulp when the
double sum sits next to a float rounding boundary; ranks are then checked through the oracle's
scores.  Against the FP64 oracle every score is within 1e-6 * max(score, 1) (scores lie in
[0, 2]; near 0 the bound is absolute).
"""
import numpy as np
import pytest

import rapidbow_b200 as rbw
from tests.helpers import random_tree

pytestmark = pytest.mark.gpu


def _ulp(x):
    return np.spacing(np.abs(np.float32(x))).astype(np.float64)


def make_docs(n_docs, n_leaves, seed, lo=20, hi=600, zipf=0.8):
    """Documents with log-uniform sizes; leaves drawn from a skewed popularity so some posting
    lists are long, with repeated leaves inside documents (tf > 1)."""
    rng = np.random.default_rng(seed)
    pop = 1.0 / np.arange(1, n_leaves + 1) ** zipf
    pop = pop[rng.permutation(n_leaves)]
    pop /= pop.sum()
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), n_docs)).astype(np.int64)
    docs = []
    for s in sizes:
        d = rng.choice(n_leaves, size=s, p=pop).astype(np.uint32)
        rep = np.nonzero(rng.random(s) < 0.1)[0]
        rep = rep[rep > 0]
        d[rep] = d[rep - 1]
        docs.append(d)
    return docs


def make_queries(docs, n_leaves, n, seed):
    rng = np.random.default_rng(seed)
    qs = []
    for i in range(n):
        if i % 3 == 2:
            qs.append(rng.integers(0, n_leaves, size=int(rng.integers(5, 400)), dtype=np.uint32))
            continue
        base = docs[int(rng.integers(0, len(docs)))]
        keep = base[rng.random(base.size) < 0.7]
        extra = rng.integers(0, n_leaves, size=max(1, base.size // 3), dtype=np.uint32)
        q = np.concatenate([keep, extra]).astype(np.uint32)
        qs.append(q[rng.permutation(q.size)])
    return qs


def build_pair(oracle, B, L, docs, ids, seed=0):
    centers, masks, weights = random_tree(B, L, seed, dup_rate=0.0)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    odb = oracle.db(B, L, weights)
    for i, d in zip(ids, docs):
        db.add_doc(int(i), d)
        odb.add(int(i), d)
    return voc, db, odb, weights


def check_query(db, odb, q, k):
    docs, scores = db.query(q, k, with_scores=True)
    odocs, oscores = odb.query(q, k, mode=0)
    assert docs.size == min(k, odocs.size)
    if docs.size == 0:
        return docs, scores
    oscore = dict(zip(odocs.tolist(), oscores.tolist()))
    # every returned document is a touched one, with the reference-arithmetic score
    mine = np.array([oscore[int(d)] for d in docs])
    assert np.all(np.abs(scores.astype(np.float64) - mine) <= _ulp(mine)), "score differs by more than 1 ulp"
    assert np.all(np.diff(scores) >= 0)
    if not np.array_equal(docs, odocs[: docs.size]):
        # allowed only where the oracle's scores at the differing ranks are within one ulp
        diff = np.nonzero(docs != odocs[: docs.size])[0]
        assert np.all(np.abs(mine[diff] - oscores[diff]) <= _ulp(oscores[diff])), "ranking differs"
    # FP64 oracle: 1e-6 * max(score, 1)
    fdocs, fscores = odb.query(q, k, mode=1)
    f = dict(zip(fdocs.tolist(), fscores.tolist()))
    ref64 = np.array([f[int(d)] for d in docs])
    assert np.all(np.abs(scores - ref64) <= 1e-6 * np.maximum(ref64, 1.0))
    return docs, scores


@pytest.mark.parametrize("B,L,n_docs", [(16, 2, 120), (16, 3, 400), (10, 4, 300), (16, 4, 600)])
def test_postings_norms_and_queries(oracle, B, L, n_docs):
    n_leaves = B ** L
    docs = make_docs(n_docs, n_leaves, seed=B * 10 + L)
    rng = np.random.default_rng(7)
    ids = rng.permutation(np.arange(n_docs, dtype=np.uint32) * 3 + 5)  # sparse, unordered ids
    _, db, odb, _ = build_pair(oracle, B, L, docs, ids)
    assert db.info() == (n_docs, sum(d.size for d in docs))
    # postings are exact (sorted ids with duplicates, as the reference stores them)
    touched = np.unique(np.concatenate(docs))
    for leaf in np.concatenate([touched[:: max(1, touched.size // 200)], [0, n_leaves - 1]]):
        assert np.array_equal(db.postings(int(leaf)), odb.postings(int(leaf)))
    # norms are bit-exact
    for i in ids[:50]:
        assert np.float32(db.doc_rcp(int(i))) == np.float32(odb.doc_rcp(int(i)))
    for k in (1, 10, 50, 1024):
        for q in make_queries(docs, n_leaves, 12, seed=k):
            check_query(db, odb, q, k)


@pytest.mark.parametrize("kind", ["idf_clamped", "wide_spread", "tiny_only_upper"])
def test_norms_bit_exact_for_every_weight_spread(oracle, kind):
    """Document and query norms are the reference's in-order double sums for every spread of
    weights: idf weights with the FLT_MIN clamp of common words (the block's exact sum sets the
    tiny terms aside), weights 2^-30 apart among the others (the in-order fallback), and words
    whose every upper level is clamped."""
    B, L = 10, 3
    rng = np.random.default_rng(61)
    centers, masks, weights = random_tree(B, L, 62, dup_rate=0.0)
    fmin = np.float32(np.finfo(np.float32).tiny)
    if kind == "idf_clamped":
        weights = np.log(rng.uniform(1.0, 5e4, weights.shape)).astype(np.float32)
        weights[:1 + B] = fmin                       # levels 0 and 1: in every document
        weights[rng.random(weights.shape) < 0.05] = fmin
    elif kind == "wide_spread":
        weights = rng.uniform(0.5, 12.0, weights.shape).astype(np.float32)
        weights[rng.random(weights.shape) < 0.3] = np.float32(3e-9)
    else:
        weights[:1 + B] = fmin
        weights[rng.random(weights.shape) < 0.5] = fmin
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    odb = oracle.db(B, L, weights)
    docs = make_docs(300, B ** L, seed=63, lo=1, hi=3000)
    for i, d in enumerate(docs):
        db.add_doc(i, d)
        odb.add(i, d)
    for i in range(len(docs)):
        assert np.float32(db.doc_rcp(i)) == np.float32(odb.doc_rcp(i)), i
    for q in make_queries(docs, B ** L, 12, seed=64):
        check_query(db, odb, q, 25)


def test_documents_touched_only_through_clamped_words_are_results(oracle):
    """A document that shares with the query only words whose idf is clamped to FLT_MIN gets
    terms that round to zero in the fixed-point sum; it is still a result (score 2), as in the
    reference, when fewer than k documents are touched."""
    B, L = 10, 3
    centers, masks, weights = random_tree(B, L, 71, dup_rate=0.0)
    fmin = np.float32(np.finfo(np.float32).tiny)
    weights = np.full(weights.shape, 2.0, dtype=np.float32)
    weights[:1 + B] = fmin                  # every upper-level word
    n_leaves = B ** L
    clamped = np.arange(0, 40, dtype=np.uint32)
    weights[(1 + B) + clamped // B, clamped % B] = fmin
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    odb = oracle.db(B, L, weights)
    docs = [
        np.array([3, 7, 7, 12], dtype=np.uint32),          # clamped words only
        np.array([5, 39, 500, 501], dtype=np.uint32),      # clamped words and others
        np.array([520, 530, 999], dtype=np.uint32),        # a normal word shared with the query
        np.array([700, 701, 702], dtype=np.uint32),        # upper-level words only in common
        np.array([3], dtype=np.uint32),                     # one clamped word
    ]
    for i, d in enumerate(docs):
        db.add_doc(i, d)
        odb.add(i, d)
    for q in (np.array([3, 7, 12, 530], dtype=np.uint32), np.array([3, 5], dtype=np.uint32),
              np.array([7, 7, 7], dtype=np.uint32)):
        got, scores = check_query(db, odb, q, 10)
        odocs, _ = odb.query(q, 10, mode=0)
        assert sorted(got.tolist()) == sorted(odocs.tolist())


def test_self_query_ranks_itself_first(oracle):
    B, L = 16, 3
    docs = make_docs(200, B ** L, seed=3)
    ids = np.arange(200, dtype=np.uint32)
    _, db, odb, _ = build_pair(oracle, B, L, docs, ids)
    for i in (0, 17, 199):
        got, scores = check_query(db, odb, docs[i], 5)
        # rank 0 is the image itself; its score is not 0 because the skip rule leaves out the
        # upper levels whose subtrees hold many postings (DataBase.cpp:125)
        assert got[0] == i and scores[0] < scores[1]


def test_matches_reference_database(oracle, reference):
    """The reference's own DataBase (compiled from its sources) returns the same ranking."""
    B, L = 16, 3
    docs = make_docs(500, B ** L, seed=11)
    ids = np.arange(500, dtype=np.uint32) + 1000
    _, db, odb, weights = build_pair(oracle, B, L, docs, ids)
    rdb = reference.db(L, weights)
    for i, d in zip(ids, docs):
        rdb.add(int(i), d)
    for k in (5, 50):
        for q in make_queries(docs, B ** L, 20, seed=100 + k):
            got = db.query(q, k)
            want = rdb.query(q, k)
            assert got.size == want.size
            if np.array_equal(got, want):
                continue
            # the reference's std::sort leaves equal scores in any order: compare through scores
            odocs, oscores = odb.query(q, k, mode=0)
            s = dict(zip(odocs.tolist(), oscores.tolist()))
            a = np.array([s[int(x)] for x in got])
            b = np.array([s[int(x)] for x in want])
            assert np.all(np.abs(a - b) <= _ulp(b))


def test_query_and_add_sequence(oracle):
    """queryAndAddDoc (DataBase.cpp:192-197) in a loop: each query sees exactly the documents
    added before it, so the index is rebuilt between calls."""
    B, L = 16, 3
    docs = make_docs(60, B ** L, seed=5)
    centers, masks, weights = random_tree(B, L, 1, dup_rate=0.0)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    odb = oracle.db(B, L, weights)
    for i, d in enumerate(docs):
        got = db.query_and_add_doc(i, d, 8)
        odocs, oscores = odb.query(d, 8, mode=0)
        odb.add(i, d)
        assert got.size == min(8, odocs.size)
        if not np.array_equal(got, odocs[: got.size]):
            s = dict(zip(odocs.tolist(), oscores.tolist()))
            a = np.array([s[int(x)] for x in got])
            assert np.all(np.abs(a - oscores[: got.size]) <= _ulp(oscores[: got.size]))
    assert db.info()[0] == 60


def test_batched_equals_single(oracle):
    import torch

    B, L = 16, 3
    docs = make_docs(300, B ** L, seed=21)
    ids = np.arange(300, dtype=np.uint32)
    _, db, odb, _ = build_pair(oracle, B, L, docs, ids)
    qs = make_queries(docs, B ** L, 37, seed=9)
    qs[3] = np.zeros(0, np.uint32)  # empty query: no results
    k = 20
    offs = np.zeros(len(qs) + 1, np.int64)
    offs[1:] = np.cumsum([q.size for q in qs])
    leaves = torch.from_numpy(np.concatenate(qs).astype(np.int32)).cuda()
    offsets = torch.from_numpy(offs).cuda()
    bd, bs, bc = db.query_batched(leaves, offsets, k)
    torch.cuda.synchronize()
    bd, bs, bc = bd.cpu().numpy().view(np.uint32), bs.cpu().numpy(), bc.cpu().numpy()
    assert bc[3] == 0
    for i, q in enumerate(qs):
        d, s = db.query(q, k, with_scores=True)
        assert bc[i] == d.size
        assert np.array_equal(bd[i, : d.size], d)
        assert np.array_equal(bs[i, : d.size], s)


def test_batched_ignores_out_of_range_leaves(oracle):
    import torch

    B, L = 16, 2
    docs = make_docs(50, B ** L, seed=2)
    _, db, _, _ = build_pair(oracle, B, L, docs, np.arange(50, dtype=np.uint32))
    q = docs[4][:30]
    bad = np.concatenate([q, np.array([B ** L, 0xFFFFFFFF, B ** L + 7], np.uint32)])
    leaves = torch.from_numpy(bad.view(np.int32)).cuda()
    offsets = torch.tensor([0, bad.size], dtype=torch.int64).cuda()
    bd, bs, bc = db.query_batched(leaves, offsets, 10)
    torch.cuda.synchronize()
    d, s = db.query(q, 10, with_scores=True)
    assert int(bc[0]) == d.size
    assert np.array_equal(bd[0, : d.size].cpu().numpy().view(np.uint32), d)
    assert np.array_equal(bs[0, : d.size].cpu().numpy(), s)


def test_many_documents_use_global_accumulators(oracle):
    """More documents than fit the in-shared-memory accumulators (20480)."""
    B, L = 16, 3
    rng = np.random.default_rng(4)
    n_docs = 25000
    docs = make_docs(n_docs, B ** L, seed=8, lo=3, hi=40)
    ids = rng.permutation(n_docs).astype(np.uint32)
    centers, masks, weights = random_tree(B, L, 2, dup_rate=0.0)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    offs = np.zeros(n_docs + 1, np.uint64)
    offs[1:] = np.cumsum([d.size for d in docs])
    db.add_docs(ids, np.concatenate(docs), offs)
    odb = oracle.db(B, L, weights)
    for i, d in zip(ids, docs):
        odb.add(int(i), d)
    for q in make_queries(docs, B ** L, 8, seed=1):
        check_query(db, odb, q, 50)
    # k above the shared-memory selection (1024): shard candidates and the merge in global memory
    for q in make_queries(docs, B ** L, 3, seed=2):
        check_query(db, odb, np.concatenate([q, np.arange(0, B ** L, 7, dtype=np.uint32)]), 1500)


@pytest.mark.parametrize("layout", [1, 2])
def test_shard_tables_and_single_table_match_oracle(oracle, layout):
    """Both inverted-file layouts (grouped tables per 2,560-document shard, one CSR per segment),
    with a main segment over 16 shards and a delta segment that straddles a shard boundary;
    results, postings and upper-level (virtual) inverted files match the oracle.  Batched
    queries (scoring CTAs over 1 to 8 shards, by batch size) equal the single queries."""
    import torch

    from rapidbow_b200 import autotune as at

    B, L = 16, 3
    n_main, n_delta = 39000, 3000
    docs = make_docs(n_main + n_delta, B ** L, seed=41, lo=2, hi=30, zipf=1.0)
    centers, masks, weights = random_tree(B, L, 42, dup_rate=0.0)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    at.clear()
    try:
        for bkt in range(32):
            at.set_value("db_shard_tables", B, L, bkt, layout)
        db = rbw.DataBase(voc)
        odb = oracle.db(B, L, weights)

        def add(lo, hi):
            offs = np.zeros(hi - lo + 1, np.uint64)
            offs[1:] = np.cumsum([d.size for d in docs[lo:hi]])
            db.add_docs(np.arange(lo, hi, dtype=np.uint32), np.concatenate(docs[lo:hi]), offs)
            for i in range(lo, hi):
                odb.add(i, docs[i])

        add(0, n_main)
        qs = make_queries(docs[:n_main], B ** L, 6, seed=43)
        # a query of rare leaves: upper-level words pass the skip rule
        qs.append(np.concatenate([docs[n_main - 1], docs[5], docs[30000]]))
        for q in qs:
            check_query(db, odb, q, 40)
        assert db.segments() == (n_main, 0)
        add(n_main, n_main + n_delta)  # slots 39000..41999: shards 15 and 16
        qs.append(np.concatenate([docs[n_main + 2999], docs[40960]]))
        for q in qs:
            check_query(db, odb, q, 40)
        check_query(db, odb, np.concatenate([qs[0], np.arange(0, B ** L, 5, dtype=np.uint32)]), 1200)
        assert db.segments() == (n_main, n_delta)
        for leaf in {int(docs[0][0]), int(docs[20480][0]), int(docs[n_main + 1500][0]), int(docs[41999][-1])}:
            assert np.array_equal(db.postings(leaf), odb.postings(leaf))
        for nq in (3, 40, 200):
            bq = make_queries(docs, B ** L, nq, seed=44 + nq)
            offs = np.zeros(nq + 1, np.int64)
            offs[1:] = np.cumsum([q.size for q in bq])
            bd, bs, bc = db.query_batched(torch.from_numpy(np.concatenate(bq).astype(np.int32)).cuda(),
                                          torch.from_numpy(offs).cuda(), 30)
            torch.cuda.synchronize()
            bd, bs, bc = bd.cpu().numpy().view(np.uint32), bs.cpu().numpy(), bc.cpu().numpy()
            for i in range(0, nq, max(1, nq // 10)):
                d, sc = check_query(db, odb, bq[i], 30)
                assert bc[i] == d.size and np.array_equal(bd[i, : d.size], d)
                assert np.array_equal(bs[i, : d.size], sc)
    finally:
        at.clear()


def test_large_documents_queries_and_result_sets(oracle):
    """Documents and queries above 32,768 descriptors (sorted in global memory) and k = 2,000
    (selected in global memory) against the oracle, single and batched; the reference's
    DataBase takes any size (DataBase.cpp:39-69,71-190)."""
    import torch

    B, L = 16, 3
    n_leaves = B ** L
    rng = np.random.default_rng(62)
    docs = make_docs(2600, n_leaves, seed=61, lo=20, hi=300)
    big = [rng.integers(0, n_leaves, 40000, dtype=np.uint32), rng.integers(0, n_leaves, 70001, dtype=np.uint32)]
    big[0][:5000] = docs[7][0]  # a long run of one leaf (tf = 5000+)
    docs = docs + big
    ids = np.arange(len(docs), dtype=np.uint32)
    _, db, odb, _ = build_pair(oracle, B, L, docs, ids)
    for i in (len(docs) - 2, len(docs) - 1):
        assert np.float32(db.doc_rcp(int(i))) == np.float32(odb.doc_rcp(int(i)))
    leaf = int(docs[7][0])
    assert np.array_equal(db.postings(leaf), odb.postings(leaf))
    qs = [np.concatenate([docs[-1][:30000], rng.integers(0, n_leaves, 15000, dtype=np.uint32)]),
          docs[5], rng.integers(0, n_leaves, 40000, dtype=np.uint32), docs[-2]]
    for q in qs:
        for k in (2000, 50):
            check_query(db, odb, q, k)
    k = 2000
    offs = np.zeros(len(qs) + 1, np.int64)
    offs[1:] = np.cumsum([q.size for q in qs])
    leaves = torch.from_numpy(np.concatenate(qs).astype(np.int32)).cuda()
    bd, bs, bc = db.query_batched(leaves, torch.from_numpy(offs).cuda(), k)
    torch.cuda.synchronize()
    bd, bs, bc = bd.cpu().numpy().view(np.uint32), bs.cpu().numpy(), bc.cpu().numpy()
    for i, q in enumerate(qs):
        d, s = db.query(q, k, with_scores=True)
        assert bc[i] == d.size == min(k, len(docs))
        assert np.array_equal(bd[i, : d.size], d)
        assert np.array_equal(bs[i, : d.size], s)


def test_edge_cases(oracle):
    B, L = 16, 2
    centers, masks, weights = random_tree(B, L, 3, dup_rate=0.0)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    # empty database
    assert db.query(np.array([1, 2, 3], np.uint32), 10).size == 0
    db.add_doc(7, np.array([5, 5, 5, 9], np.uint32))
    db.add_doc(0xFFFFFFF0, np.array([9, 200], np.uint32))
    db.add_doc(3, np.zeros(0, np.uint32))  # empty document: no postings
    with pytest.raises(rbw.RbwError) as e:
        db.add_doc(7, np.array([1], np.uint32))
    assert e.value.status == rbw.RBW_ERR_DUPLICATE
    with pytest.raises(rbw.RbwError) as e:
        db.add_doc(8, np.array([B ** L], np.uint32))
    assert e.value.status == rbw.RBW_ERR_INVALID_ARG
    with pytest.raises(rbw.RbwError):
        db.add_docs(np.array([20, 20], np.uint32), np.array([1, 2], np.uint32), np.array([0, 1, 2], np.uint64))
    assert db.info() == (3, 6)
    assert np.array_equal(db.postings(5), [7, 7, 7])
    assert np.array_equal(db.postings(9), [7, 0xFFFFFFF0])
    assert db.query(np.array([5], np.uint32), 0).size == 0
    got = db.query(np.array([9, 5], np.uint32), 10)
    odb = oracle.db(B, L, weights)
    odb.add(7, np.array([5, 5, 5, 9], np.uint32))
    odb.add(0xFFFFFFF0, np.array([9, 200], np.uint32))
    odb.add(3, np.zeros(0, np.uint32))
    odocs, _ = odb.query(np.array([9, 5], np.uint32), 10)
    assert np.array_equal(got, odocs[:10])
    # adding after a query rebuilds the index
    db.add_doc(11, np.array([9, 9], np.uint32))
    assert 11 in db.query(np.array([9, 9], np.uint32), 10).tolist()
    # max_results beyond every touched document: all of them (no limit on k)
    odb.add(11, np.array([9, 9], np.uint32))
    odocs, _ = odb.query(np.array([9, 5], np.uint32), 5000)
    assert np.array_equal(db.query(np.array([9, 5], np.uint32), 5000), odocs)
    assert odocs.size == 3


def test_incremental_segments_match_oracle(oracle):
    """Adds after queries go to the delta segment, which is merged into the main segment once it
    outgrows max(256, main / 4) documents; results match the oracle at every step."""
    B, L = 16, 3
    docs = make_docs(900, B ** L, seed=31, lo=10, hi=200)
    centers, masks, weights = random_tree(B, L, 6, dup_rate=0.0)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    odb = oracle.db(B, L, weights)
    qs = make_queries(docs, B ** L, 6, seed=4)

    def add(lo, hi):
        for i in range(lo, hi):
            db.add_doc(i, docs[i])
            odb.add(i, docs[i])

    add(0, 300)
    for q in qs:
        check_query(db, odb, q, 20)
    assert db.segments() == (300, 0)       # 300 > 256: first update builds the main segment
    add(300, 310)
    for q in qs:
        check_query(db, odb, q, 20)
    assert db.segments() == (300, 10)      # small delta
    for i in range(310, 330):              # query-and-add loop: one document per update
        got = db.query_and_add_doc(i, docs[i], 5)
        od, _ = odb.query(docs[i], 5)
        odb.add(i, docs[i])
        assert got.size == min(5, od.size)
    assert db.segments()[0] == 300
    add(330, 620)                           # delta 320 > max(256, 75): merged
    check_query(db, odb, qs[0], 50)
    assert db.segments() == (620, 0)
    leaf = int(docs[5][0])
    assert np.array_equal(db.postings(leaf), odb.postings(leaf))
    add(620, 900)
    for q in qs:
        check_query(db, odb, q, 1024)
    for i in (0, 450, 899):
        assert np.float32(db.doc_rcp(i)) == np.float32(odb.doc_rcp(i))


def test_batched_queries_interleaved_with_adds(oracle):
    """Batched queries on a user stream and adds on the host thread need no synchronisation:
    each batch sees the documents added before it was issued."""
    import torch

    B, L = 16, 2
    docs = make_docs(120, B ** L, seed=12, lo=5, hi=80)
    centers, masks, weights = random_tree(B, L, 9, dup_rate=0.0)
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    odb = oracle.db(B, L, weights)
    q = docs[3][:40]
    leaves = torch.from_numpy(q.astype(np.int32)).cuda()
    offsets = torch.tensor([0, q.size], dtype=torch.int64).cuda()
    stream = torch.cuda.Stream()
    outs = []
    for step in range(4):
        for i in range(step * 30, step * 30 + 30):
            db.add_doc(i, docs[i])
            odb.add(i, docs[i])
        with torch.cuda.stream(stream):
            outs.append(db.query_batched(leaves, offsets, 10, stream=stream))
        want, _ = odb.query(q, 10)
        outs[-1] = (outs[-1], want[:10].copy())
    torch.cuda.synchronize()
    for (d, s, c), want in outs:
        assert int(c[0]) == want.size
        assert set(d[0, : want.size].cpu().numpy().view(np.uint32).tolist()) == set(want.tolist())
