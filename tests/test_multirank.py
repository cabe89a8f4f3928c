"""The multi-GPU path of the bench is replicas (one member per rank, no collective on the data path): the job's step
time is the max over ranks and its value the sum over replicas. Checked here with two gloo ranks on CPU (no GPU)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(1.0 + rank, dist, 'cpu')      # rank 1 is the slow one
        q.put((rank, ms, bench.job_value(world, 300.0, ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_and_sum_replicas():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.0, 2.0]
    # two replicas, each 300 s of model time per 2 ms step: 2 * (300 / 86400) / 0.002 model days/s
    assert out[0][2] == pytest.approx(2 * (300.0 / 86400.0) / 0.002)


def test_single_process_passes_through():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, None, 'cpu') == 3.5
    assert bench.job_value(1, 300.0, 1.0) == pytest.approx(300.0 / 86400.0 / 1e-3)
