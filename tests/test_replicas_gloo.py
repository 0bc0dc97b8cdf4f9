"""World-size-2 check of the replica bench's cross-rank reduction (gloo on CPU)."""

import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


def test_bench_starts_its_own_ranks():
    """``bench.py --gpus 2`` without a torchrun environment starts two ranks itself; the
    printed line counts both and takes the slower rank's time (gloo, no GPU work)."""
    import json
    import subprocess
    import sys

    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--launch-check"],
                         capture_output=True, text=True, timeout=240, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["n_gpus"] == 2 and line["parallelism"] == "replicas x2"
    assert line["ms_per_step"] >= 19.0 and line["ms_per_step"] >= line["rank0_ms"]


def test_bench_rejects_a_world_size_other_than_gpus():
    import subprocess
    import sys

    env = dict(os.environ, WORLD_SIZE="3", RANK="0", LOCAL_RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--launch-check"],
                         capture_output=True, text=True, timeout=120, env=env, cwd=ROOT)
    assert out.returncode != 0 and "WORLD_SIZE=3" in out.stderr
