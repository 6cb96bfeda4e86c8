"""The N>1 path of bench.py on CPU: two gloo ranks, replicas with distinct
workload seeds, timing aggregated as the max over ranks (no data-path
collective exists: ciphertexts are independent)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 100.0 + 50.0 * rank            # rank 1 is the slow one
        total = bench.max_over_ranks(local_ms, dist, "cpu")
        seed = bench.rank_seed(7, rank)
        seeds = [None] * world
        dist.all_gather_object(seeds, seed)
        q.put((rank, total, seeds))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, total, seeds in res:
        assert total == 150.0                     # max over ranks
        assert len(set(seeds)) == 2               # independent replicas
