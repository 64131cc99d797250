"""The N > 1 plumbing of bench.py on CPU: two gloo ranks, barrier and max-over-ranks timing.
The lookup shards descriptors across ranks with the tree replicated, so no collective touches
the data path; only the timing is reduced."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        bench.barrier(world)
        got = bench.allreduce_max(world, 1.5 + rank)  # each rank's own step time
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 2.5, 1: 2.5}
