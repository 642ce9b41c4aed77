"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1) run the
same helpers the GPU ranks use — the max-over-ranks reduction of the timed
region, the barrier, and the per-rank replica workloads (each rank solves
its own operator: different potential seeds, no data-path collective)."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from nutrlan_b200 import operators as ops
        # Timed-region reduction: every rank gets the slowest rank's time.
        t = bench.reduce_max(dist, 0.5 + rank, torch.device("cpu"))
        bench.barrier(dist)
        # Replica workloads: the Anderson replica of each rank differs.
        w = bench.WORKLOADS["anderson128"]
        A = ops.anderson_3d(8, W=w["W"], seed=2024 + rank)
        d = float(A.val[A.row_ptr[0]:A.row_ptr[1]][A.col[A.row_ptr[0]:A.row_ptr[1]] == 0][0])
        all_d = [None] * world
        dist.all_gather_object(all_d, d)
        q.put((rank, t, all_d))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_replicate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res = dict((r, (t, d)) for r, t, d in out)
    assert res[0][0] == res[1][0] == 1.5          # max over ranks
    d0, d1 = res[0][1]
    assert d0 != d1                                # distinct replicas
