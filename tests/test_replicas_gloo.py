"""The multi-rank path on CPU (gloo, world size 2): work assignment and the
max-over-ranks timing used by bench.py and the serving loop."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from ocfd_b200.replicas import assign, max_over_ranks, sum_over_ranks

    mine = assign(range(10), rank, world)
    t = max_over_ranks(1.0 + rank)
    n = sum_over_ranks(len(mine))
    out[rank] = (mine, t, n)
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_world2():
    import torch.multiprocessing as mp

    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    assert out[0][0] == [0, 2, 4, 6, 8] and out[1][0] == [1, 3, 5, 7, 9]
    assert out[0][1] == out[1][1] == 2.0
    assert out[0][2] == out[1][2] == 10.0
