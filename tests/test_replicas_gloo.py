"""Multi-rank host logic of the benchmark on CPU: world size 2 over gloo.  Each rank solves its
own replica (the path has no collective inside a solve); the benchmark reduces time with max
and work with sum over ranks."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from _util import ROOT  # noqa: F401  (puts the repository on sys.path)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = 100.0 + 50.0 * rank          # rank 1 is slower
    work = 1000.0 * (rank + 1)
    t_max, w_sum = bench.reduce_ranks([(ms, "max"), (work, "sum")], dist, "cpu")
    q.put((rank, t_max, w_sum))
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, t_max, w_sum in res:
        assert t_max == 150.0
        assert w_sum == 3000.0


def test_reduce_without_group_is_identity():
    import bench
    assert bench.reduce_ranks([(3.0, "max"), (4.0, "sum")], None, "cpu") == [3.0, 4.0]
