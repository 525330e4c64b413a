"""The replica path of bench.py on the host: two gloo ranks (127.0.0.1)
agree on the max-over-ranks timing that the N-GPU bench reports."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v = bench.max_over_ranks(torch, dist, 10.0 + rank)
        q.put((rank, v))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: 11.0, 1: 11.0}


def test_max_over_ranks_single_process():
    import torch
    import bench
    assert bench.max_over_ranks(torch, None, 3.5) == 3.5
