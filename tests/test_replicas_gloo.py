"""Multi-rank path of bench.py on CPU (gloo, world size 2).

Isotherm points are independent fixed-point problems, so multi-GPU runs are
replicas: each rank solves its own isotherm and the only collective is the
reduction of two scalars after the timed region (max of the device time,
sum of converged points).  This runs that reduction under gloo.
"""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    ms, n = bench.reduce_over_ranks(10.0 + 5.0 * rank, 21, world, "cpu")
    out.put((rank, ms, n))
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_over_ranks_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, n in res:
        assert ms == 15.0      # max over ranks of 10 and 15 ms
        assert n == 42.0       # 21 converged points per replica


def test_reduce_single_rank_is_identity():
    import bench
    assert bench.reduce_over_ranks(12.5, 7, 1, "cpu") == (12.5, 7.0)
