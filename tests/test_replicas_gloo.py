"""The multi-GPU bench path runs independent replicas; its only collectives
are the max of the timed device time and the sum of the work.  Checked here
with two gloo ranks on CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms, work = (100.0 + 50.0 * rank), float(1000 * (rank + 1))
    mx, tot = bench.reduce_timing(ms, work, device="cpu")
    out[rank] = (mx, tot)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_reduction_two_ranks():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        assert out[r] == (150.0, 3000.0)
