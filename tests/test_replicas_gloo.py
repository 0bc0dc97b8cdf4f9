"""World-size-2 check of the replica bench's cross-rank reduction (gloo on CPU)."""

import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        value = bench.max_over_ranks(10.0 * (rank + 1), dist, torch.device("cpu"))
        out[rank] = value
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_gloo():
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        assert dict(out) == {0: 20.0, 1: 20.0}
