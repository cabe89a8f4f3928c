"""The mixed precision form (FP32 momentum, TRiSK operators and FCT flux corrections; FP64 thickness, masses, the fast
loop's sum and the budgets) against the plain FP64 form, which the parity tests hold to the oracle:

- the level-6 member (air 3 + ocean 2 layers, 3 tracers each) after 10 model days: relative L2 error of h and u <= 1e-5
  per stack, layer mass drift <= 1e-13 (relative, per layer) and tracer mass drift <= 1e-13; the same at levels 4, 5
  and 7 (the ensemble and serving levels), with the stacks the mixed form runs in FP64 there equal to FP64 bit for bit;
- the level-7 Galewsky jet over 6 model days: h and vertex vorticity norms against FP64, mass drift <= 1e-13;
- the per-call Layers.step of the mixed form equals the batched step bit for bit, and a stack's result is the same alone
  and batched with others (on any grid), bit for bit.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def dev():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch.device('cuda:0')


def rl2(x, y):
    return float(torch.linalg.norm(x - y) / torch.linalg.norm(y))


def member(level, precision, seed=0, ntracers=3):
    from isw import gpu
    from isw import grid as G
    from isw.batch import Batch
    from isw.workload import Member, planet_grid
    gpu.set_precision(precision)
    try:
        g = planet_grid(G.build(level, device=0))
        batch = Batch(0)
        m = Member(gpu.DeviceGrid(g), seed=seed, ntracers=ntracers, batch=batch)
    finally:
        gpu.set_precision('double')
    return m, batch


def layer_masses(stack):
    """sum_i A_i h_k,i per layer, and sum_i M_k,i psi_k,i per tracer and layer (deterministic sums)."""
    from isw.gpu import dsum
    A = torch.as_tensor(stack.dg.host.areaCell, device=stack.h.device)
    hm = [dsum(stack.h[k], A) for k in range(stack.L)]
    tm = [dsum(t[k], stack.M[k]) for t in stack.tracers for k in range(stack.L)]
    return np.array(hm), np.array(tm)


def test_level6_member_ten_days(dev):
    mm, bm = member(6, 'mixed')
    md, bd = member(6, 'double')
    m0 = [layer_masses(s) for s in mm.stacks]
    steps = int(round(10 * 86400 / mm.dt))
    for _ in range(steps):
        bm.step()
        bd.step()
    torch.cuda.synchronize()
    assert bm.status() == 0 and bd.status() == 0
    for sm, sd, (h0, t0) in zip(mm.stacks, md.stacks, m0):
        eh, eu = rl2(sm.h, sd.h), rl2(sm.u, sd.u)
        assert eh <= 1e-5 and eu <= 1e-5, (eh, eu)
        h1, t1 = layer_masses(sm)
        assert np.max(np.abs(h1 - h0) / np.abs(h0)) <= 1e-13
        assert np.max(np.abs(t1 - t0) / np.abs(t0)) <= 1e-13


@pytest.mark.parametrize('level', [4, 5, 7])
def test_member_ten_days_at_ensemble_levels(dev, level):
    """The member at the other levels the ensemble and serving configs run (4 .. 7), over 10 model days, as mixed-form
    ensembles and serving run it: relative L2 error of h and u <= 1e-5 per stack against the FP64 form, and layer-volume
    and tracer-mass drift <= 1e-13. At levels 4 and 5 the ocean stack runs in the FP64 form inside the mixed batch
    (workload.FP64_IN_MIXED: its flow amplifies FP32 rounding past 1e-5) and equals the FP64 form bit for bit."""
    from isw import accuracy
    from isw.workload import fp64_stack_kinds
    r = accuracy.member(level, 10.0)
    assert r['status'] == [0, 0]
    for row in r['stacks']:
        assert row['h_l2'] <= 1e-5 and row['u_l2'] <= 1e-5, row
        assert row['volume_drift_mixed'] <= 1e-13 and row['tracer_mass_drift_mixed'] <= 1e-13, row
        if row['stack'] in fp64_stack_kinds(level):
            assert row['form'] == 'double' and row['h_linf'] == 0 and row['u_linf'] == 0, row
        else:
            assert row['form'] == 'mixed', row


@pytest.mark.parametrize('level', [5, 6])
def test_member_ten_days_grid_wide(dev, level):
    """The member over 10 model days with the fast loop in grid-wide passes (the layout batches of several members
    run; in the mixed form its sub-step sum comes from the per-cell weighted sum of Y): the same bounds against the FP64
    form as in tiles, relative L2 of h and u <= 1e-5 and layer-volume and tracer-mass drift <= 1e-13."""
    from isw import accuracy
    r = accuracy.member(level, 10.0, tiles=False)
    assert r['status'] == [0, 0]
    for row in r['stacks']:
        assert row['h_l2'] <= 1e-5 and row['u_l2'] <= 1e-5, row
        assert row['volume_drift_mixed'] <= 1e-13 and row['tracer_mass_drift_mixed'] <= 1e-13, row


def test_level7_galewsky_six_days(dev):
    """The Galewsky jet at level 7 over the full 6 model days (9216 steps of 56.25 s), mixed form against the
    FP64 form (reference tests/test_accuracy.py:51-55 vertex vorticity, :111-128 Galewsky): relative L2 and Linf of h
    <= 1e-5, of vertex vorticity <= 1e-3 (the jet's vorticity is small-scale where the instability rolls up), and mass
    drift <= 1e-13 in both forms. The norms are printed (pytest -s)."""
    from isw import accuracy
    r = accuracy.galewsky(7, 6.0)
    print('galewsky level 7, 6 days:', r)
    assert r['steps'] == 9216 and r['status'] == [0, 0]
    assert r['h_l2'] <= 1e-5 and r['h_linf'] <= 1e-5, r
    assert r['vorticity_l2'] <= 1e-3 and r['vorticity_linf'] <= 1e-3, r
    assert abs(r['mass_drift_mixed']) <= 1e-13 and abs(r['mass_drift_double']) <= 1e-13, r


def test_percall_mixed_equals_batched(dev, grid4):
    from isw import gpu
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import planet_grid
    from isw import cases
    gpu.set_precision('mixed')
    try:
        dg = DeviceGrid(planet_grid(grid4))
        from isw.workload import Stack
        s = cases.stack_state(dg.host, 'air', 0, ntracers=0)
        a = Stack(dg, s, 450.0, 20, ntracers=0)
        b = Stack(dg, s, 450.0, 20, ntracers=0)
    finally:
        gpu.set_precision('double')
    batch = Batch(0)
    b.register(batch)
    for _ in range(8):
        a.core.step(a.h, a.u, a.dt, a.nfast, a.Fm)
        batch.step()
    torch.cuda.synchronize()
    assert torch.equal(a.h, b.h) and torch.equal(a.u, b.u) and torch.equal(a.Fm, b.Fm)


def test_mixed_alone_equals_in_a_mix(dev):
    alone, ba = member(5, 'mixed', seed=3, ntracers=2)
    mix, bm = member(5, 'mixed', seed=3, ntracers=2)
    others = [member(4, 'mixed', seed=7, ntracers=2)]
    # put the other member's stacks into the mixed batch too
    for s in others[0][0].stacks:
        s.register(bm)
    for _ in range(12):
        ba.step()
        bm.step()
    torch.cuda.synchronize()
    for x, y in zip(alone.state(), mix.state()):
        assert torch.equal(x, y)
