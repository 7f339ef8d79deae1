"""bench.py's multi-GPU path is replicas only (no collective on the data path):
the timing is the maximum over ranks.  Checked with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = 10.0 * (rank + 1)               # each replica reports its own time
    out[rank] = bench.max_over_ranks(ms, dist)
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
