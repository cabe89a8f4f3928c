"""Parity at the benchmark's full size. The level-6 member (an air stack of 3 layers and an ocean stack of 2, 3 FCT
tracers each, nfast 20, dt 300 s) is advanced one model day (288 steps) by the batched CUDA step and by the CPU oracle
from the same state: every field within 1e-12 of the oracle's, relative to the field's largest value (the stress terms
call exp(), whose last bit may differ between the host's libm and CUDA). The level-7 Galewsky jet (one layer, no
exp()) is held bit for bit over 96 steps."""
import sys

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def dev():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from isw import gpu
    gpu.set_precision('double')
    return torch.device('cuda:0')


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_level6_member_one_model_day(dev, oracle_lib):
    sys.path.insert(0, str(ROOT))
    import bench
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    g = planet_grid(G.build(6, device=0))
    batch = Batch(0)
    m = Member(DeviceGrid(g), seed=0, batch=batch)
    cpu_step, dt = bench.cpu_member(g, 0, 'oracle')
    steps = int(round(86400 / dt))
    assert steps == 288
    for _ in range(steps):
        batch.step()
    torch.cuda.synchronize()
    assert batch.status() == 0
    for _ in range(steps):
        cpu_step()
    errs = [rel(x.cpu().numpy(), y) for x, y in zip(m.state(), cpu_step.state())]
    assert len(errs) == 2 * 6
    assert max(errs) <= 1e-12, errs


def test_level7_galewsky_bit_exact(dev, oracle_lib):
    from isw import cases
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.layers import Layers
    g = G.for_planet(G.build(7, device=0), 6.371e6, 7.292e-5, 9.80616)
    h0, b, u0 = cases.initial_state(g, 'galewsky')
    dt, nfast = cases.default_dt(7), 2
    core = Layers(DeviceGrid(g), 1, b=b)
    h = torch.as_tensor(np.ascontiguousarray(h0[None]), device=dev)
    u = torch.as_tensor(np.ascontiguousarray(u0[None]), device=dev)
    batch = Batch(0)
    batch.add(core, h, u, torch.zeros_like(u), dt=dt, nfast=nfast)
    M = oracle_lib
    oc = M.Layers(M.OracleGrid(g), 1, b=b)
    oh, ou, oF = h0[None].copy(), u0[None].copy(), np.zeros_like(u0[None])
    for _ in range(96):
        batch.step()
        oc.step(oh, ou, dt, nfast, oF)
    torch.cuda.synchronize()
    assert batch.status() == 0
    assert np.array_equal(h.cpu().numpy(), oh)
    assert np.array_equal(u.cpu().numpy(), ou)
