"""Ensembles and the serving loop in the mixed form: a member of an ensemble of mixed grid levels ends bit for bit where
it ends alone, and a served request's result is the same whether it was served alone or admitted into a running mix of
other requests (continuous batching: requests join and leave the batch between steps)."""
import math

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def dev():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch.device('cuda:0')


@pytest.fixture(scope='module')
def grids(dev):
    from isw import gpu
    from isw.ensemble import device_grids
    gpu.set_precision('mixed')
    try:
        return device_grids([4, 5], 0)
    finally:
        gpu.set_precision('double')


def test_ensemble_member_equals_alone(dev, grids):
    from isw.ensemble import Ensemble
    ens = Ensemble.build([4, 5, 4, 5], seed=40, ntracers=2, precision='mixed', grids=grids)
    alone = Ensemble.build([5], seed=41, ntracers=2, precision='mixed', grids=grids)
    assert len(ens) == 4 and ens.member_days_per_step() > 0
    ens.step(6)
    alone.step(6)
    torch.cuda.synchronize()
    assert ens.batch.status() == 0
    for x, y in zip(ens.members[1].state(), alone.members[0].state()):
        assert torch.equal(x, y)


def test_served_alone_equals_in_mix(dev, grids):
    from isw.serving import Request, Server
    target = Request(0, 0.0, 5, 0.1, 5, seed=77)
    others = [Request(1, 0.0, 4, 0.3, 3, seed=78), Request(2, 0.0, 5, 0.05, 3, seed=79),
              Request(3, 0.02, 4, 0.2, 5, seed=80), Request(4, 0.05, 5, 0.15, 3, seed=81)]
    res = {}
    for name, reqs in (('alone', [target]), ('mix', [others[0], target] + others[1:])):
        srv = Server(0, budget_bytes=150e9, precision='mixed', ntracers=2, grids=grids, keep_state=True)
        srv.batch.config(layout='packed')
        results, stats = srv.run(reqs)
        assert stats['requests'] == len(reqs)
        assert srv.batch.status() == 0
        for r in results:
            assert r.done >= r.admitted >= r.arrival >= 0
            assert r.steps == max(1, math.ceil(r.days * 86400 / (1200.0 * 2.0 ** (4 - r.level)) - 1e-9))
        res[name] = next(r for r in results if r.rid == 0)
    assert res['alone'].steps == res['mix'].steps
    for x, y in zip(res['alone'].state, res['mix'].state):
        assert torch.equal(x, y)


def test_admission_respects_budget(dev, grids):
    """With a budget that holds one request at a time, requests are served one after another (never two active)."""
    from isw.serving import Request, Server
    reqs = [Request(i, 0.0, 4, 0.05, 3, seed=90 + i) for i in range(3)]
    srv = Server(0, budget_bytes=1.0, precision='mixed', ntracers=2, grids=grids)
    results, stats = srv.run(reqs)
    assert [r.rid for r in results] == [0, 1, 2]
    for a, b in zip(results, results[1:]):
        assert b.admitted >= a.done - 1e-3


def test_checkpoint_resume_equals_uninterrupted(dev, grids, tmp_path):
    """A served request stopped after 5 batched steps, checkpointed (reference save-file format) and resumed in a new
    server ends bit for bit where the uninterrupted run ends; a request still waiting at the checkpoint runs too."""
    from isw.serving import Request, Server
    def reqs():
        return [Request(0, 0.0, 4, 0.25, 5, seed=61), Request(1, 0.0, 5, 0.1, 3, seed=62)]
    whole = Server(0, precision='mixed', ntracers=2, grids=grids, keep_state=True)
    first = Server(0, precision='mixed', ntracers=2, grids=grids, budget_bytes=1.0)   # one resident at a time
    again = Server(0, precision='mixed', ntracers=2, grids=grids, keep_state=True)
    for srv in (whole, first, again):
        srv.batch.config(layout='packed')          # every stack in tiles, whatever shares the batch
    ref = {r.rid: r for r in whole.run(reqs())[0]}
    done, _ = first.run(reqs(), stop_after=5, checkpoint_dir=tmp_path)
    assert not done and (tmp_path / 'manifest.json').exists()
    res = {r.rid: r for r in again.run(Server.resume(tmp_path))[0]}
    assert sorted(res) == [0, 1]
    for rid in (0, 1):
        assert res[rid].steps == ref[rid].steps
        for x, y in zip(res[rid].state, ref[rid].state):
            assert torch.equal(x, y)


def test_nonfinite_request_dropped_others_complete(dev, grids):
    """A request whose state goes non-finite (a NaN planted in its initial thickness, on the host) is dropped with an
    error result after its first step; the batch's status is cleared and the other requests complete with the same
    results as when served without it, bit for bit."""
    import numpy as np
    from isw import cases
    from isw.serving import Request, Server

    def reqs(with_bad):
        out = [Request(0, 0.0, 4, 0.1, 5, seed=71), Request(2, 0.0, 5, 0.05, 3, seed=73)]
        if with_bad:
            g = grids[4].host
            topo = cases.topography(g, 72)
            bad = Request(1, 0.0, 4, 0.2, 3, seed=72)
            bad.state = [cases.stack_state(g, 'air', 72, perturb=0.01, ntracers=2, topo=topo)]
            bad.state[0]['h'][1, 17] = np.nan
            out.insert(1, bad)
        return out
    res = {}
    for name in ('clean', 'with_bad'):
        srv = Server(0, budget_bytes=150e9, precision='mixed', ntracers=2, grids=grids, keep_state=True)
        srv.batch.config(layout='packed')
        results, stats = srv.run(reqs(name == 'with_bad'))
        assert srv.batch.status() == 0
        res[name] = {r.rid: r for r in results}
        if name == 'with_bad':
            assert stats['failed'] == 1 and stats['requests'] == 2
            assert res[name][1].error.startswith('non-finite thickness after 1 steps')
    for rid in (0, 2):
        assert not res['with_bad'][rid].error
        for x, y in zip(res['clean'][rid].state, res['with_bad'][rid].state):
            assert torch.equal(x, y)


def test_reused_member_equals_fresh(dev, grids):
    """A request admitted into the member a finished request of the same kind left behind (its state, terrain and
    tracers loaded into it) ends bit for bit where it ends in a fresh server."""
    from isw.serving import Request, Server

    def run(reqs, budget):
        srv = Server(0, budget_bytes=budget, precision='mixed', ntracers=2, grids=grids, keep_state=True)
        res, _ = srv.run(reqs)
        assert srv.batch.status() == 0
        return {r.rid: r for r in res}, srv
    first = Request(0, 0.0, 4, 0.2, 5, seed=91)
    second = Request(1, 0.0, 4, 0.1, 5, seed=92)
    both, srv = run([first, second], 1.0)                 # one resident at a time: the second reuses the first's member
    assert sum(len(v) for v in srv._pool.values()) == 1 and both[1].admitted >= both[0].done - 1e-3
    alone, _ = run([Request(1, 0.0, 4, 0.1, 5, seed=92)], 150e9)
    assert both[1].steps == alone[1].steps
    for x, y in zip(both[1].state, alone[1].state):
        assert torch.equal(x, y)
