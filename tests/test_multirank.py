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


def test_plain_gpus_2_call_starts_two_ranks():
    """`bench.py --gpus 2` without torchrun starts the two ranks itself (torch.distributed.run on 127.0.0.1); their
    plumbing runs on gloo here: rank 0 prints one line for the whole job, with the slowest rank's time."""
    import json
    import subprocess
    env = dict(os.environ)
    for k in ('WORLD_SIZE', 'RANK', 'LOCAL_RANK', 'MASTER_ADDR', 'MASTER_PORT'):
        env.pop(k, None)
    r = subprocess.run([sys.executable, str(ROOT / 'bench.py'), '--gpus', '2', '--plumbing'], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith('{')]
    assert len(lines) == 1
    d = lines[0]
    assert d['n_gpus'] == 2
    assert d['ms_per_step'] >= d['rank_ms']                 # rank 0 ran the shorter loop; the job takes the max
    assert d['value'] == pytest.approx(2 * (300.0 / 86400.0) / (d['ms_per_step'] / 1e3))


def test_rank_count_must_match_gpus():
    import subprocess
    env = dict(os.environ, WORLD_SIZE='1', RANK='0', LOCAL_RANK='0')
    r = subprocess.run([sys.executable, str(ROOT / 'bench.py'), '--gpus', '2', '--plumbing'], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and '1 ranks for --gpus 2' in r.stderr
