"""Multi-GPU timing logic of bench.py on CPU: replicas (independent
projections per rank, no data-path collective), the max over ranks of the
timed region, whole-job ms per projection. Two gloo ranks stand in for GPUs."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, elapsed, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    v = bench.job_ms_per_projection(elapsed[rank], steps=5, world=world, device="cpu")
    out[rank] = v
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_max_over_ranks(world):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    elapsed = [10.0, 20.0]
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, world, port, elapsed, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    # slowest rank (20 ms) over 5 projections x 2 ranks
    assert out[0] == out[1] == pytest.approx(20.0 / 10)


def test_single_rank_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_ms_per_projection(12.0, steps=4, world=1) == 3.0
