"""Multi-rank path of bench.py on CPU: two gloo ranks, one process each.

The N>1 bench runs independent replicas (the path does not shard) and
reports the slowest rank's timings; this checks the max-over-ranks reduction
and that every rank takes the same collective steps, without a GPU.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # per-rank timings: rank r is slower in a different entry each
        local = np.array([10.0 + rank, 5.0 - rank, 1.0 + 0.5 * rank, 2.0], np.float64)
        out = bench.reduce_max_over_ranks(local, torch.device("cpu"))
        dist.barrier()
        q.put((rank, out.tolist(), local.tolist()))
    finally:
        dist.destroy_process_group()


def test_reduce_max_over_ranks_gloo_world2():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = np.max([np.array(local) for _, _, local in res], axis=0)
    for rank, out, _ in res:
        np.testing.assert_array_equal(np.array(out), expect)


def test_reduce_max_identity_single_process():
    sys.path.insert(0, ROOT)
    import torch

    import bench
    v = np.array([3.0, 1.0])
    np.testing.assert_array_equal(bench.reduce_max_over_ranks(v, torch.device("cpu")), v)
