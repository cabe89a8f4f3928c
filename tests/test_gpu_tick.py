"""The reference's callers' step sequences with the isw core inside, on a B200, against the CPU oracle running the same
sequence (the reference's kernels restated; pinned to the reference's own golden vectors elsewhere).

- The ocean's step (reference ocean.py:247-252): core.step(h, u, 3600, nfast, Fm), mass_after, step_many([T, S]),
  M <- M1, with the ocean's own layer parameters (ocean.py:30-35, 88-90: three layers 100 / 600 / 3300 m over a 4 km
  basin, g' 0.016, floor 10 m, nabla^4 from visc4_U 0.5, bottom stress 2.5e-4, interfacial stress 5e-4 with the Earth
  preset's quadratic part 1e-3, thin 2).
- The world's tick (world.py:286-301, 360-383): step, mass_after, step_many over the moved tracers, M <- M1; the first
  tick direct, then the tick captured once as a CUDA graph on the world's stream and replayed, which must equal direct
  ticks bit for bit (the reference's REPRO: graph vs direct), for Boussinesq layers and for air layers with theta."""
import math

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

REL = 1e-12          # the stress terms call exp, whose last bit may differ between the host's libm and CUDA


@pytest.fixture(scope='module')
def dev():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch.device('cuda:0')


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def T(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)


def ocean_case(g, seed=3):
    """Three ocean layers at rest but for a 0.3 m/s barotropic jet and a 5% seeded thickness perturbation; T, S."""
    from isw import cases
    rng = np.random.default_rng(seed)
    H = np.array([100.0, 600.0, 3300.0])
    noise = 1 + 0.05 * cases.smooth_noise(g, seed)
    h = np.stack([H[k] * noise for k in range(3)])
    lat_e, _, en, _ = cases.edge_east_north(g)
    u = np.stack([0.3 * np.cos(lat_e) * en] * 3)
    Tt = np.stack([293.0 + 5 * rng.random(g.N), 283.0 + rng.random(g.N), 274.0 + 0.1 * rng.random(g.N)])
    S = 35.0 + 0.5 * rng.random((3, g.N))
    return h, u, Tt, S, np.full(g.N, -4000.0)


def test_ocean_step_sequence(dev, oracle_lib, grid4):
    """Twelve hourly ocean steps through isw equal the oracle's to 1e-12 (h, u, M, T, S), and M stays the mass the
    transport carried (M <- M1 each step)."""
    from isw import cases
    from isw import grid as G
    from isw.gpu import DeviceGrid, set_precision
    from isw.layers import Layers
    from isw.transport import Transport
    M_ = oracle_lib
    set_precision('double')
    g = G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616)
    h0, u0, T0, S0, b = ocean_case(g)
    kw = dict(b=b, gprime=[0.016, 0.016], stress=[0.0, 0.0, 2.5e-4], nu4=cases.visc4(g, 0.5), floor=10.0, vmix=5e-4,
              vmix_cd=1e-3, thin=2.0)
    dg = DeviceGrid(g)
    core, tr = Layers(dg, 3, **kw), Transport(dg, layers=3, tracers=2)
    nfast = core.substeps(T(h0, dev), 3600.0)
    h, u, Tt, S = T(h0, dev), T(u0, dev), T(T0, dev), T(S0, dev)
    A = T(g.areaCell, dev)
    M, M1, Fm = (h * A[None]).contiguous(), torch.zeros_like(h), torch.zeros_like(u)
    og = M_.OracleGrid(g)
    oc, ot = M_.Layers(og, 3, **kw), M_.Transport(og, layers=3, tracers=2)
    assert oc.substeps(h0, 3600.0) == nfast
    oh, ou, oT, oS = h0.copy(), u0.copy(), T0.copy(), S0.copy()
    oM, oM1, oF = oh * g.areaCell[None], np.zeros_like(oh), np.zeros_like(ou)
    for _ in range(12):
        core.step(h, u, 3600.0, nfast, Fm)
        tr.mass_after(M, Fm, M1)
        tr.step_many(M, M1, Fm, [Tt, S], order=3)
        M.copy_(M1)
        oc.step(oh, ou, 3600.0, nfast, oF)
        ot.mass_after(oM, oF, oM1)
        ot.step_many(oM, oM1, oF, [oT, oS], order=3)
        oM[...] = oM1
    torch.cuda.synchronize()
    for name, x, y in (('h', h, oh), ('u', u, ou), ('M', M, oM), ('T', Tt, oT), ('S', S, oS)):
        assert rel(x.cpu().numpy(), y) <= REL, name
    assert np.allclose(M.cpu().numpy(), oh * g.areaCell[None], rtol=0, atol=1e-6 * np.max(oM))


def _world_tick(core, tr, st, dt, nfast, theta=None):
    h, u, M, M1, Fm, moved = st
    core.step(h, u, dt, nfast, Fm, theta=theta)
    tr.mass_after(M, Fm, M1)
    tr.step_many(M, M1, Fm, moved, order=3)
    M.copy_(M1)


def _world_state(h0, u0, tracers, area, dev):
    h, u = T(h0, dev), T(u0, dev)
    M = (h * area[None]).contiguous()
    moved = [T(t, dev) for t in tracers]
    return [h, u, M, torch.zeros_like(M), torch.zeros_like(u), moved]


def test_world_tick_graph_equals_direct_and_oracle(dev, oracle_lib, grid4):
    """The reference's three-layer stacked golden case as a world tick with one tracer: a first direct tick, then the
    tick captured once on the world's stream and replayed 11 times, equals 12 direct ticks bit for bit, and both equal
    the oracle's ticks to 1e-12."""
    from isw import grid as G
    from isw.gpu import DeviceGrid, set_precision
    from isw.layers import Layers
    from isw.transport import Transport
    M_ = oracle_lib
    set_precision('double')
    z = golden('air3_n4')
    g = G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616)
    kw = dict(b=z['b'], gprime=list(z['gprime']), stress=list(z['stress']), nu4=float(z['nu4']), floor=float(z['floor']),
              vmix=float(z['vmix']))
    dt, nfast = float(z['dt']), int(z['nfast'])
    dg = DeviceGrid(g)
    A = T(g.areaCell, dev)
    psi0 = np.stack([np.linspace(0.0, 1.0, g.N)] * 3) + 0.1 * np.arange(3)[:, None]
    direct = (Layers(dg, 3, **kw), Transport(dg, layers=3), _world_state(z['h0'], z['u0'], [psi0], A, dev))
    graphed = (Layers(dg, 3, **kw), Transport(dg, layers=3), _world_state(z['h0'], z['u0'], [psi0], A, dev))
    for _ in range(12):
        _world_tick(direct[0], direct[1], direct[2], dt, nfast)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        _world_tick(graphed[0], graphed[1], graphed[2], dt, nfast)       # the first tick runs directly
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            _world_tick(graphed[0], graphed[1], graphed[2], dt, nfast)
    for _ in range(11):
        graph.replay()
    torch.cuda.synchronize()
    for a, b in zip(direct[2][:3] + direct[2][5], graphed[2][:3] + graphed[2][5]):
        assert torch.equal(a, b)
    og = M_.OracleGrid(g)
    oc, ot = M_.Layers(og, 3, **kw), M_.Transport(og, layers=3)
    oh, ou, opsi = z['h0'].copy(), z['u0'].copy(), psi0.copy()
    oM, oM1, oF = oh * g.areaCell[None], np.zeros_like(oh), np.zeros_like(ou)
    for _ in range(12):
        oc.step(oh, ou, dt, nfast, oF)
        ot.mass_after(oM, oF, oM1)
        ot.step_many(oM, oM1, oF, [opsi], order=3)
        oM[...] = oM1
    for name, x, y in (('h', direct[2][0], oh), ('u', direct[2][1], ou), ('M', direct[2][2], oM), ('psi', direct[2][5][0], opsi)):
        assert rel(x.cpu().numpy(), y) <= REL, name


def test_air_world_tick_graph_equals_direct(dev, grid4):
    """Air layers (h = mass per area, theta moved by the transport with the tracer, as world.py:293-301 does): 12 direct
    ticks equal one direct tick and 11 replays of the captured tick, bit for bit."""
    from isw import grid as G
    from isw.gpu import DeviceGrid, set_precision
    from isw.layers import Layers
    from isw.transport import Transport
    set_precision('double')
    z = golden('airtheta_n4')
    g = G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616)
    dg = DeviceGrid(g)
    A = T(g.areaCell, dev)
    air = dict(t_ref=288.0, cp=float(z['cp']), kappa=float(z['kappa']), rd=float(z['rd']))
    L = int(z['h0'].shape[0])
    kw = dict(b=z['b'], gprime=[0.0] * (L - 1), stress=list(z['stress']), nu4=float(z['nu4']), floor=float(z['floor']),
              vmix=float(z['vmix']), air=air)
    psi0 = np.stack([np.linspace(0.0, 1.0, g.N)] * L)
    worlds = []
    for _ in range(2):
        core, tr = Layers(dg, L, **kw), Transport(dg, layers=L, tracers=2)
        st = _world_state(z['h0'], z['u0'], [psi0, z['theta0']], A, dev)
        core.update_gfast(st[0], st[5][1])
        worlds.append((core, tr, st))
    dt, nfast = float(z['dt']), int(z['nfast'])
    core, tr, st = worlds[0]
    for _ in range(12):
        _world_tick(core, tr, st, dt, nfast, theta=st[5][1])
    core, tr, st = worlds[1]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        _world_tick(core, tr, st, dt, nfast, theta=st[5][1])
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            _world_tick(core, tr, st, dt, nfast, theta=st[5][1])
    for _ in range(11):
        graph.replay()
    torch.cuda.synchronize()
    a, b = worlds[0][2], worlds[1][2]
    for x, y in zip(a[:3] + a[5], b[:3] + b[5]):
        assert torch.equal(x, y)
    assert all(bool(torch.isfinite(x).all()) for x in a[:3] + a[5])
