"""The multi-GPU data path on CPU ranks (gloo, world size 2): the sharded k-means build moves
per-node sums, counts, change counts, initial rows and child sizes between ranks and must give
the single-rank build byte for byte; the sharded inverted file all-reduces the skip-rule counts
and all-gathers per-shard top-k lists, and must give the single database's top-k exactly.

The per-rank compute here is the oracle (numpy + oracle/liborc.so) behind the same engine
interface as the GPU engine (rapidbow_b200.distributed.CudaShardEngine); the driver, the
collectives and the merge are the product code."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class OracleShardEngine:
    """One rank's descriptors, assign/update/regroup by the oracle (kmeans.cu semantics, IEEE
    division), with the GPU engine's interface and buffer layouts."""

    def __init__(self, desc, B, oracle):
        import torch

        self.desc = np.ascontiguousarray(desc, np.uint8)
        self.n_local = self.desc.shape[0]
        self.B = B
        self.orc = oracle
        self.device = torch.device("cpu")
        self.groups = [np.arange(self.n_local, dtype=np.uint32)]
        self.assigns = [np.zeros(self.n_local, np.uint8)]
        self.centers = None

    def node_counts(self):
        return np.array([g.size for g in self.groups], np.uint32)

    def member_rows(self, nodes, pos):
        return self.desc[[int(self.groups[int(n)][int(p)]) for n, p in zip(nodes, pos)]]

    def desc_rows(self, idx):
        return self.desc[np.asarray(idx, np.int64)]

    def set_centers(self, c):
        self.centers = np.array(c, np.uint8)
        self.assigns = [np.zeros(g.size, np.uint8) for g in self.groups]

    def buffers(self, nb):
        import torch

        return (torch.zeros(nb, dtype=torch.int32), torch.zeros((nb, 16, 128), dtype=torch.int64),
                torch.zeros((nb, 16), dtype=torch.int32), torch.zeros(nb, dtype=torch.int32))

    def assign(self, last, sums, counts, changed):
        B = self.B
        for g, members in enumerate(self.groups):
            if int(last[g]) == 0:
                continue
            a, cnt, s, ch = self.orc.kmeans_assign(self.desc, members, self.centers[g], B, self.assigns[g])
            self.assigns[g] = a
            counts[g, :B] += np.asarray(cnt, np.int64).astype(np.int32)
            sums[g, :B] += np.asarray(s, np.int64)
            changed[g] += ch

    def update(self, sums, counts, changed):
        B = self.B
        for g in range(len(self.groups)):
            if int(changed[g]) != 0:
                self.centers[g] = self.orc.kmeans_update(counts[g, :B].numpy().astype(np.uint32),
                                                         sums[g, :B].numpy().astype(np.uint64), self.centers[g])

    def get_centers(self):
        return self.centers.copy()

    def next_level(self):
        groups, child = [], []
        for g, members in enumerate(self.groups):
            for b in range(self.B):
                sel = members[self.assigns[g] == b]
                groups.append(sel)
                child.append(sel.size)
        self.groups = groups
        return np.array(child, np.uint32)


def _data():
    from rapidbow_b200.synth import sift_like

    return sift_like(20000, seed=71, n_components=4096, zipf=1.1).numpy()


def _rank_build(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from oracle.pyoracle import Oracle, level_beg
    from rapidbow_b200.distributed import build_vocabulary_sharded

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        desc = _data()
        cut = [0, 7000, desc.shape[0]]  # uneven shards
        B, L = 10, 3
        eng = OracleShardEngine(desc[cut[rank]: cut[rank + 1]], B, Oracle())
        c, m, w = build_vocabulary_sharded(eng, B, L, 500, init="reference", max_iterations=10)
        rng = np.random.default_rng(3)
        inj = rng.integers(0, desc.shape[0], (level_beg(B, L), B)).astype(np.uint32)
        inj[rng.random(inj.shape[0]) < 0.1, -1] = 0xFFFFFFFF
        eng2 = OracleShardEngine(desc[cut[rank]: cut[rank + 1]], B, Oracle())
        c2, m2, w2 = build_vocabulary_sharded(eng2, B, L, 500, init="injected", injected=inj, max_iterations=10,
                                              check_interval=3)
        q.put((rank, c, m, w, c2, m2, w2, inj))
    finally:
        dist.destroy_process_group()


def test_sharded_build_equals_single_rank_build(oracle):
    from oracle.pyoracle import INIT_INJECTED, INIT_REFERENCE

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_build, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=300)
        res[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    desc = _data()
    ref = oracle.build_vocabulary(desc, 500, 10, 3, max_iter=10, init=INIT_REFERENCE)
    ref2 = oracle.build_vocabulary(desc, 500, 10, 3, max_iter=10, init=INIT_INJECTED, injected=res[0][6])
    for r in (0, 1):
        c, m, w, c2, m2, w2, _ = res[r]
        assert np.array_equal(c, ref["centers"]) and np.array_equal(m, ref["masks"])
        assert np.array_equal(w, ref["weights"])
        assert np.array_equal(c2, ref2["centers"]) and np.array_equal(m2, ref2["masks"])
        assert np.array_equal(w2, ref2["weights"])


class OracleDbShard:
    """The oracle DataBase behind the DataBase interface ShardedDataBase uses."""

    def __init__(self, odb):
        self.odb = odb

    def add_doc(self, i, leaves):
        self.odb.add(i, leaves)

    def query(self, leaves, k, with_scores=True):
        d, s = self.odb.query(leaves, k, mode=0)
        return d[:k], s[:k].astype(np.float32)

    def word_postings(self):
        return self.odb.word_postings()

    def set_word_postings(self, counts):
        self.odb.set_word_postings(counts)


def _db_case():
    from tests.helpers import random_tree
    from tests.test_database_gpu import make_docs, make_queries

    B, L = 16, 3
    docs = make_docs(120, B ** L, seed=81, lo=40, hi=160)
    qs = make_queries(docs, B ** L, 16, seed=82)
    _, _, weights = random_tree(B, L, 83, dup_rate=0.0)
    return B, L, docs, qs, weights


def _rank_db(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from oracle.pyoracle import Oracle
    from rapidbow_b200.distributed import ShardedDataBase

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        B, L, docs, qs, weights = _db_case()
        shard = ShardedDataBase(OracleDbShard(Oracle().db(B, L, weights)))
        lo, hi = (0, 50) if rank == 0 else (50, len(docs))  # document-range shards
        for i in range(lo, hi):
            shard.add_doc(i, docs[i])
        unsynced = [shard.query(x, 3) for x in qs]
        shard.sync()
        out = [(k, [shard.query(x, k) for x in qs]) for k in (3, 10, 200)]
        q.put((rank, out, unsynced))
    finally:
        dist.destroy_process_group()


def test_sharded_database_topk_equals_single_database(oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_db, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=300)
        res[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    B, L, docs, qs, weights = _db_case()
    odb = oracle.db(B, L, weights)
    for i, d in enumerate(docs):
        odb.add(i, d)
    differs_unsynced = 0
    for r in (0, 1):
        out, unsynced = res[r]
        for k, results in out:
            for x, (gd, gs) in zip(qs, results):
                wd, ws = odb.query(x, k, mode=0)
                assert np.array_equal(gd, wd[:k]), (k, gd[:5], wd[:5])
                assert np.array_equal(gs, ws[:k].astype(np.float32))
        for x, (gd, gs) in zip(qs, unsynced):
            wd, ws = odb.query(x, 3, mode=0)
            differs_unsynced += int(not (np.array_equal(gd, wd[:3]) and np.array_equal(gs, ws[:3].astype(np.float32))))
    # without the global counts the shards apply the skip rule to their own postings only
    assert differs_unsynced > 0
