"""Multi-rank host logic on CPU (gloo, world size 2): the bench's max-over-ranks
device-time reduction and the per-rank replica seeding used for weak scaling."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    out[rank] = (bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu"), bench.replica_seed(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_seeds():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    assert res[0][1] != res[1][1]


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
