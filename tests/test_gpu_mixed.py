"""The mixed precision form (FP32 momentum, TRiSK operators and FCT flux corrections; FP64 thickness, masses, the fast
loop's sum and the budgets) against the plain FP64 form, which the parity tests hold to the oracle:

- the level-6 member (air 3 + ocean 2 layers, 3 tracers each) after 10 model days: relative L2 error of h and u <= 1e-5
  per stack, layer mass drift <= 1e-13 (relative, per layer) and tracer mass drift <= 1e-13;
- the level-7 Galewsky jet for 0.5 model day: h and vertex vorticity close to FP64, mass drift <= 1e-13;
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


def test_level7_galewsky_half_day(dev):
    from isw import cases, gpu
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid, dsum
    from isw.layers import Layers
    g = G.for_planet(G.build(7, device=0), 6.371e6, 7.292e-5, 9.80616)
    h0, b, u0 = cases.initial_state(g, 'galewsky')
    dt, nfast = cases.default_dt(7), 2
    A = torch.as_tensor(g.areaCell, device=dev)
    out = {}
    for prec in ('mixed', 'double'):
        gpu.set_precision(prec)
        try:
            core = Layers(DeviceGrid(g), 1, b=b)
        finally:
            gpu.set_precision('double')
        h = torch.as_tensor(np.ascontiguousarray(h0[None]), device=dev)
        u = torch.as_tensor(np.ascontiguousarray(u0[None]), device=dev)
        batch = Batch(0)
        batch.add(core, h, u, torch.zeros_like(u), dt=dt, nfast=nfast)
        mass0 = dsum(h[0], A)
        for _ in range(768):                           # half a model day
            batch.step()
        torch.cuda.synchronize()
        assert batch.status() == 0
        out[prec] = (h, u, core, abs(dsum(h[0], A) - mass0) / mass0)
    hm, um, core, drift = out['mixed']
    hd, ud, _, _ = out['double']
    assert drift <= 1e-13
    assert rl2(hm, hd) <= 1e-6
    assert rl2(um, ud) <= 1e-4


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
