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


def test_bench_spawns_its_own_ranks():
    """`bench.py --gpus 2` started without a launcher reruns itself under
    torch.distributed.run with two ranks; here the ranks join a gloo group on
    the host and rank 0 reports the world size and the max over ranks."""
    import json
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(repo, "bench.py"), "--gpus", "2", "--replica-check"],
                       capture_output=True, text=True, timeout=240, env=env, cwd=repo)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert lines == [{"replica_check": True, "n_gpus": 2, "max_ms": 11.0}], r.stdout


def test_reference_arm_loads_no_cuda_library():
    """The CPU arms classify the cells with the oracle: building the bench
    case for them maps no part of libhsolver_b200.so into the process."""
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import bench\n"
            "bench.workload('config1', host_side=True)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'liboracle' in maps\n"
            "print('libhsolver_b200' in maps)\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=240, cwd=repo)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == "False"
