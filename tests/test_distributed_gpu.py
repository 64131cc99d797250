"""The multi-GPU data path with the GPU engines: two ranks (processes) that share one GPU and
exchange data through gloo on the host -- no kernel of one rank waits for the other.  The
sharded build (rbw_kmeans_shard_*) must equal the one-GPU build with IEEE center rounding byte
for byte, and the sharded DataBase (rbw_db_* with the summed skip-rule counts) must give the
single database's top-k, ids and scores."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _spawn(fn, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=fn, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r = q.get(timeout=600)
        res[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return res


def _init(rank, world, port):
    import datetime

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(0)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))


def _desc():
    from rapidbow_b200.synth import sift_like

    return sift_like(300_000, seed=101, n_components=4096, zipf=1.1).numpy()


def _rank_build(rank, world, port, q):
    import torch
    import torch.distributed as dist

    from rapidbow_b200.distributed import CudaShardEngine, build_vocabulary_sharded

    _init(rank, world, port)
    try:
        desc = _desc()
        cut = [0, 120_000, desc.shape[0]]
        local = torch.from_numpy(desc[cut[rank]: cut[rank + 1]]).cuda()
        eng = CudaShardEngine(local, 16, 3)
        c, m, w = build_vocabulary_sharded(eng, 16, 3, 1000, init="reference", max_iterations=10)
        q.put((rank, c, m, w))
    finally:
        dist.destroy_process_group()


def test_sharded_gpu_build_equals_one_gpu_build(oracle):
    import torch

    import rapidbow_b200 as rbw

    res = _spawn(_rank_build)
    desc = _desc()
    voc = rbw.build_vocabulary(torch.from_numpy(desc).cuda(), 16, nb_doc=1000, nb_levels=3, init="reference",
                               max_iterations=10, ieee_division=True)
    c, m, w = voc.tree()
    for r in (0, 1):
        rc, rm, rw = res[r]
        assert np.array_equal(rc, c) and np.array_equal(rm, m) and np.array_equal(rw, w)


def _db_case():
    from tests.helpers import random_tree
    from tests.test_database_gpu import make_docs, make_queries

    B, L = 16, 3
    docs = make_docs(400, B ** L, seed=111, lo=40, hi=300)
    qs = make_queries(docs, B ** L, 20, seed=112)
    centers, masks, weights = random_tree(B, L, 113, dup_rate=0.0)
    return B, L, docs, qs, centers, masks, weights


def _rank_db(rank, world, port, q):
    import torch.distributed as dist

    import rapidbow_b200 as rbw
    from rapidbow_b200.distributed import ShardedDataBase

    _init(rank, world, port)
    try:
        B, L, docs, qs, centers, masks, weights = _db_case()
        voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
        shard = ShardedDataBase(rbw.DataBase(voc))
        for i in range(rank, len(docs), world):  # documents dealt round-robin
            shard.add_doc(i, docs[i])
        shard.sync()
        q.put((rank, [(k, [shard.query(x, k) for x in qs]) for k in (3, 20, 300)]))
    finally:
        dist.destroy_process_group()


def test_sharded_gpu_database_equals_single_database():
    import rapidbow_b200 as rbw

    res = _spawn(_rank_db)
    B, L, docs, qs, centers, masks, weights = _db_case()
    voc = rbw.vocabulary_from_host(B, L, centers, masks, weights)
    db = rbw.DataBase(voc)
    for i, d in enumerate(docs):
        db.add_doc(i, d)
    for r in (0, 1):
        for k, results in res[r][0]:
            for x, (gd, gs) in zip(qs, results):
                wd, ws = db.query(x, k, with_scores=True)
                assert np.array_equal(gd, wd) and np.array_equal(gs, ws)
