"""Host-side logic of the N-GPU replica benchmark, run as two gloo ranks on
the CPU: time = max over ranks, rays = sum over ranks."""
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
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t, c = bench.reduce_over_ranks(dist, "cpu", 10.0 + 5.0 * rank, 1000 * (rank + 1))
        q.put((rank, t, c))
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, t, c in got:
        assert t == 15.0            # slowest rank's time
        assert c == 3000.0          # rays of both replicas


def test_reduce_over_ranks_single_process():
    import bench
    assert bench.reduce_over_ranks(None, "cpu", 2.5, 7) == (2.5, 7.0)
