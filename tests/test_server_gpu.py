"""The continuous-batching server: every result equals the one the same request gets alone and
the one of a direct lookup + query; batching, overlap and memory admission behave as stated."""
import threading

import numpy as np
import pytest
import torch

import rapidbow_b200 as rbw
from rapidbow_b200.synth import sift_like

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    train = sift_like(60_000, seed=3, device="cuda")
    voc = rbw.build_vocabulary(train, 16, nb_doc=300, nb_levels=3, init="kmeans++", seed=1, max_iterations=8)
    rng = np.random.default_rng(0)
    sizes = rng.integers(50, 600, size=300)
    pool = sift_like(int(sizes.sum()) + 40 * 700, seed=9).numpy()
    leaves = voc.lookup(torch.from_numpy(pool).cuda()).cpu().numpy().view(np.uint32)
    db = rbw.DataBase(voc)
    off = 0
    for i, s in enumerate(sizes):
        db.add_doc(i, leaves[off: off + s])
        off += int(s)
    # query images: half are subsets of database images' descriptors, half fresh, uneven sizes
    queries = []
    for j in range(40):
        s = int(rng.integers(1, 700))
        if j % 2 == 0:
            d = int(rng.integers(0, 300))
            beg = int(sizes[:d].sum())
            take = min(s, int(sizes[d]))
            queries.append(pool[beg: beg + take].copy())
        else:
            queries.append(pool[off: off + s].copy())
            off += s
    queries.append(np.zeros((0, 128), np.uint8))  # an empty image
    return voc, db, queries


def direct(voc, db, q, k):
    if q.shape[0] == 0:
        return np.zeros(0, np.uint32), np.zeros(0, np.float32)
    leaves = voc.lookup(torch.from_numpy(q).cuda()).cpu().numpy().view(np.uint32)
    return db.query(leaves, k, with_scores=True)


def test_alone_equals_mix_equals_direct(setup):
    voc, db, queries = setup
    k = 20
    srv = rbw.Server(voc, db, max_results=k)
    alone = []
    for q in queries:
        rid = srv.submit(q)
        alone.append(srv.wait(rid)[:2])
    st = srv.stats()
    assert st["completed"] == len(queries) and st["mean_batch_requests"] == 1.0

    # the mix: all submitted at once from two threads, collected out of order
    srv.reset_stats()
    ids = [None] * len(queries)

    def feeder(idx):
        for i in idx:
            ids[i] = srv.submit(queries[i])

    ts = [threading.Thread(target=feeder, args=(range(p, len(queries), 2),)) for p in (0, 1)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    mixed = {}
    for i in reversed(range(len(queries))):
        d, s, lat = srv.wait(ids[i])
        assert lat >= 0
        mixed[i] = (d, s)
    st = srv.stats()
    assert st["completed"] == len(queries)
    assert st["batches"] < len(queries)          # requests were batched together
    for i, q in enumerate(queries):
        dd, ds = direct(voc, db, q, k)
        assert np.array_equal(alone[i][0], dd) and np.array_equal(alone[i][1], ds)
        assert np.array_equal(mixed[i][0], dd) and np.array_equal(mixed[i][1], ds)
    srv.close()


def test_memory_budget_limits_batches(setup):
    voc, db, queries = setup
    k = 10
    big = [q for q in queries if q.shape[0] > 300][:6]
    sizes = [q.shape[0] for q in big]
    probe = rbw.Server(voc, db, max_results=k)
    one = max(probe.batch_bytes(n, 1) for n in sizes)
    two = min(probe.batch_bytes(a + b, 2) for i, a in enumerate(sizes) for b in sizes[i + 1:])
    small = min(probe.batch_bytes(n, 1) for n in sizes)
    probe.close()
    assert two > one + 1024 and small > 1024
    # a budget that admits exactly one of these requests at a time
    srv = rbw.Server(voc, db, max_results=k, hbm_budget_bytes=one + 1024)
    ids = [srv.submit(q) for q in big]
    res = [srv.wait(i)[:2] for i in ids]
    st = srv.stats()
    assert st["batches"] == len(big) and st["max_inflight_seen"] == 1
    for (d, s), q in zip(res, big):
        dd, ds = direct(voc, db, q, k)
        assert np.array_equal(d, dd) and np.array_equal(s, ds)
    with pytest.raises(rbw.RbwError) as e:
        srv.submit(np.zeros((20000, 128), np.uint8))
    assert e.value.status == rbw.RBW_ERR_OUT_OF_MEMORY
    srv.close()


def test_overlap_and_errors(setup):
    voc, db, queries = setup
    srv = rbw.Server(voc, db, max_results=5, max_batch_queries=4, max_inflight_batches=3)
    ids = [srv.submit(q) for q in queries for _ in range(3)]
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    assert st["max_inflight_seen"] >= 2           # batches overlapped on the GPU
    assert st["mean_batch_requests"] <= 4
    with pytest.raises(rbw.RbwError):
        srv.wait(ids[0])                          # already collected
    srv.close()
    # a request above 32,768 descriptors is served like any other (sorted in global memory)
    srv = rbw.Server(voc, db, max_results=5, max_batch_descriptors=60000)
    big = np.concatenate([queries[0]] * (40000 // queries[0].shape[0] + 1))[:40000]
    d, s, _ = srv.wait(srv.submit(big))
    dd, ds = direct(voc, db, big, 5)
    assert np.array_equal(d, dd) and np.array_equal(s, ds)
    with pytest.raises(rbw.RbwError) as e:
        srv.submit(np.zeros((60001, 128), np.uint8))  # larger than a batch
    assert e.value.status == rbw.RBW_ERR_INVALID_ARG
    srv.close()


def test_documents_added_while_serving(setup):
    voc, _, queries = setup
    db = rbw.DataBase(voc)
    q = queries[0]
    leaves = voc.lookup(torch.from_numpy(q).cuda()).cpu().numpy().view(np.uint32)
    srv = rbw.Server(voc, db, max_results=3)
    d0, _, _ = srv.wait(srv.submit(q))
    assert d0.size == 0                           # empty database
    db.add_doc(77, leaves)
    d1, s1, _ = srv.wait(srv.submit(q))
    assert d1.tolist() == [77]
    srv.close()
