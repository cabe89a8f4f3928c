"""Parity of the CUDA core with the reference, through the C ABI (isw Python facade), on a B200.

The golden vectors were produced by the reference's own Layers / Transport / dsum (tests/golden/make_golden.py). Runs
without exp() in their arithmetic must match bit for bit; runs whose stress terms call exp() may differ from the host
build in the last bit of exp, so they are held to 1e-12 relative (the FP64 bar) and are reported as bit-exact or not.
"""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

REL = 1e-12


@pytest.fixture(scope='module')
def dev():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch.device('cuda:0')


@pytest.fixture(scope='module')
def isw(dev):
    from isw import gpu, layers, transport
    gpu.set_precision('double')
    return gpu, layers, transport


def T(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_w2_bit_exact(dev, isw, grid4):
    """Williamson 2 (n = 4, dt 900 s, nfast from the reference's rule): 1, 96 and 480 steps bit for bit."""
    from isw import grid as G
    gpu, layers, _ = isw
    z = golden('w2_n4')
    dg = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, float(z['omega']), 9.80616))
    core = layers.Layers(dg, 1, b=z['b'])
    h, u = T(z['h0'], dev), T(z['u0'], dev)
    assert core.substeps(h, float(z['dt'])) == int(z['substeps'])
    for s in range(1, 481):
        core.step(h, u, float(z['dt']), int(z['nfast']))
        if s in (1, 96, 480):
            torch.cuda.synchronize()
            assert np.array_equal(h.cpu().numpy(), z[f'h{s}']), (s, rel(h.cpu().numpy(), z[f'h{s}']))
            assert np.array_equal(u.cpu().numpy(), z[f'u{s}']), (s, rel(u.cpu().numpy(), z[f'u{s}']))
    assert core.energy(h, u) == float(z['energy480'])


def run_stack(isw, grid4, z, dev, steps):
    from isw import grid as G
    gpu, layers, transport = isw
    dg = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616))
    L = int(z['L'])
    core = layers.Layers(dg, L, b=z['b'], gprime=list(z['gprime']), stress=list(z['stress']), nu4=float(z['nu4']),
                         floor=float(z['floor']), vmix=float(z['vmix']))
    tr = transport.Transport(dg, layers=L, tracers=3)
    h, u = T(z['h0'], dev), T(z['u0'], dev)
    M = T(z['h0'] * grid4.areaCell[None], dev)
    M1 = torch.zeros_like(M)
    Fm = torch.zeros_like(u)
    trc = [T(z[f'tr{k}_0'], dev) for k in range(3)]
    for _ in range(steps):
        core.step(h, u, float(z['dt']), int(z['nfast']), Fm)
        tr.mass_after(M, Fm, M1)
        tr.step_many(M, M1, Fm, trc, order=3)
        M, M1 = M1, M
    torch.cuda.synchronize()
    return core, h, u, M, trc, Fm


@pytest.mark.parametrize('case', ['air3_n4', 'ocean2_n4'])
def test_stacks_golden(dev, isw, grid4, case, record_property):
    """Stacked layers (nu4, stress, interfacial stress, 20 fast sub-steps, 3 FCT tracers), 6 steps: <= 1e-12 relative
    to the reference in every field (bit-exact where no exp() is involved)."""
    z = golden(case)
    core, h, u, M, trc, Fm = run_stack(isw, grid4, z, dev, 6)
    worst = 0.0
    exact = True
    for name, a in (('h', h), ('u', u), ('M', M), ('Fm', Fm)) + tuple((f'tr{k}', trc[k]) for k in range(3)):
        a = a.cpu().numpy()
        exact &= bool(np.array_equal(a, z[name]))
        worst = max(worst, rel(a, z[name]))
    record_property('bit_exact', exact)
    record_property('worst_rel', worst)
    assert worst <= REL, worst
    assert abs(core.lap_max() - float(z['lap_max'])) <= 1e-10 * float(z['lap_max'])


def test_outcrop_golden(dev, isw, grid4):
    """The reference's outcrop case: floor limiter active, bottom stress, nu4, bell tracer, 24 steps; <= 1e-12."""
    gpu, layers, transport = isw
    z = golden('outcrop_n4')
    dg = gpu.DeviceGrid(grid4)
    core = layers.Layers(dg, 2, b=z['b'], gprime=[0.02], stress=[0.0, 2.5e-4], nu4=float(z['nu4']), floor=1.0)
    tr = transport.Transport(dg, layers=2, tracers=4)
    h, u, psi = T(z['h0'], dev), T(z['u0'], dev), T(z['psi0'], dev)
    M = T(z['h0'] * grid4.areaCell[None], dev)
    M1, Fm = torch.zeros_like(M), torch.zeros_like(u)
    lo = float(h.min())
    for _ in range(24):
        core.step(h, u, float(z['dt']), int(z['nfast']), Fm)
        tr.mass_after(M, Fm, M1)
        tr.step_many(M, M1, Fm, [psi], order=3)
        M, M1 = M1, M
        lo = min(lo, float(h.min()))
    for name, a in (('h', h), ('u', u), ('M', M), ('psi', psi), ('Fm', Fm)):
        assert rel(a.cpu().numpy(), z[name]) <= REL, name
    assert lo >= 1.0 - 1e-9


def test_bell_bit_exact(dev, isw, grid4):
    """Transport alone (cosine bell, solid-body flux), order 1 and 3, 20 steps: bit for bit."""
    gpu, _, transport = isw
    z = golden('bell_n4')
    dg = gpu.DeviceGrid(grid4)
    for order in (1, 3):
        tr = transport.Transport(dg)
        psi, M, M1, Fm = T(z['psi0'], dev), T(z['M0'], dev), torch.zeros(1, dg.N, dtype=torch.float64, device=dev), T(z['Fm'], dev)
        for _ in range(20):
            tr.mass_after(M, Fm, M1)
            tr.step(M, M1, Fm, psi, order)
            M, M1 = M1, M
        assert np.array_equal(psi.cpu().numpy(), z[f'psi_o{order}']), order
        assert np.array_equal(M.cpu().numpy(), z[f'M_o{order}']), order


def test_dsum_bit_exact(dev, isw):
    """The deterministic tree sum equals the reference's, for sizes from 1 to 2^20, with and without y."""
    gpu = isw[0]
    z = golden('dsum')
    for n in (1, 2, 255, 2048, 2049, 100003, 1 << 20):
        i = np.arange(n, dtype=np.int64)
        x = ((i * 7919) % 10007 - 5003) / 997.0
        y = ((i * 104729) % 65521) / 4093.0
        assert gpu.dsum(T(x, dev)) == float(z[f'x_{n}'])
        assert gpu.dsum(T(x, dev), T(y, dev)) == float(z[f'xy_{n}'])


def test_reference_device_grid_accepted(dev, isw, grid4):
    """Layers and Transport built on the reference's own DeviceGrid (an object carrying the host Grid as .host, its
    precision as .mixed, and the kernel() the rest of the model compiles its other kernels with) use an isw grid made
    from that Grid once, and step exactly as on an isw DeviceGrid."""
    from isw import grid as G
    gpu, layers, transport = isw
    z = golden('w2_n4')
    g = G.for_planet(grid4, 6.371e6, float(z['omega']), 9.80616)

    class ReferenceDeviceGrid:                # the attributes the reference's DeviceGrid carries that isw reads
        def __init__(self, grid):
            self.host, self.mixed = grid, False

        def kernel(self, name, file, defs=()):
            raise AssertionError('isw compiles nothing through the caller grid')
    ref_dg = ReferenceDeviceGrid(g)
    a, b = layers.Layers(ref_dg, 1, b=z['b']), layers.Layers(gpu.DeviceGrid(g), 1, b=z['b'])
    assert a.dg is gpu.as_device_grid(ref_dg) and transport.Transport(ref_dg).dg is a.dg
    states = [(T(z['h0'], dev), T(z['u0'], dev)) for _ in range(2)]
    for core, (h, u) in zip((a, b), states):
        for _ in range(5):
            core.step(h, u, float(z['dt']), int(z['nfast']))
    torch.cuda.synchronize()
    assert torch.equal(states[0][0], states[1][0]) and torch.equal(states[0][1], states[1][1])


def test_graph_capture_equals_direct(dev, isw, grid4):
    """A step queued inside the caller's own CUDA-graph capture and replayed equals direct steps, bit for bit
    (reference REPRO: graph vs direct)."""
    from isw import grid as G
    gpu, layers, _ = isw
    z = golden('w2_n4')
    dg = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, float(z['omega']), 9.80616))
    a, b = layers.Layers(dg, 1, b=z['b']), layers.Layers(dg, 1, b=z['b'])
    ha, ua = T(z['h0'], dev), T(z['u0'], dev)
    hb, ub = ha.clone(), ua.clone()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.step(hb, ub, 900.0, 2)            # first step direct (as World does), then capture
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            b.step(hb, ub, 900.0, 2)
    torch.cuda.synchronize()
    for _ in range(10):
        g.replay()
    for _ in range(11):                     # b: one direct step and ten replays
        a.step(ha, ua, 900.0, 2)
    torch.cuda.synchronize()
    assert torch.equal(ha, hb) and torch.equal(ua, ub)
    # a first step inside the capture (the private batch cannot be built there: the per-call kernels are captured)
    c = layers.Layers(dg, 1, b=z['b'])
    hc, uc = T(z['h0'], dev), T(z['u0'], dev)
    with torch.cuda.stream(s):
        g2 = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g2, stream=s):
            c.step(hc, uc, 900.0, 2)
    torch.cuda.synchronize()
    for _ in range(11):
        g2.replay()
    torch.cuda.synchronize()
    assert torch.equal(ha, hc) and torch.equal(ua, uc)


def test_two_equal_layers_equal_one(dev, isw, grid4):
    """A one-layer case split into two equal layers with g' = 0 moves exactly as one layer (reference REPRO, layers)."""
    from isw import grid as G
    gpu, layers, _ = isw
    z = golden('w2_n4')
    dg = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, float(z['omega']), 9.80616))
    one = layers.Layers(dg, 1, b=z['b'])
    two = layers.Layers(dg, 2, b=z['b'], gprime=[0.0])
    h1, u1 = T(z['h0'], dev), T(z['u0'], dev)
    h2, u2 = T(np.repeat(z['h0'] / 2, 2, axis=0), dev), T(np.repeat(z['u0'], 2, axis=0), dev)
    for _ in range(50):
        one.step(h1, u1, 900.0, 2)
        two.step(h2, u2, 900.0, 2)
    torch.cuda.synchronize()
    assert torch.equal(h2[0], h2[1]) and torch.equal(u2[0], u2[1])
    assert torch.equal(2 * h2[0], h1[0]) and torch.equal(u2[0], u1[0])


def test_stack_conservation(dev, isw, grid4):
    """Per-layer volume and tracer mass are conserved to roundoff (reference CONSERVE bar 1e-13) over 6 steps."""
    gpu = isw[0]
    z = golden('air3_n4')
    core, h, u, M, trc, Fm = run_stack(isw, grid4, z, dev, 6)
    A = T(grid4.areaCell, dev)
    M0 = T(z['h0'] * grid4.areaCell[None], dev)
    for k in range(int(z['L'])):
        v0, v1 = gpu.dsum(M0[k]), gpu.dsum(h[k] * A)
        assert abs(v1 - v0) / v0 <= 1e-13
        t0 = gpu.dsum(M0[k], T(z['tr0_0'][k], dev))
        t1 = gpu.dsum(M[k], trc[0][k])
        assert abs(t1 - t0) / abs(t0) <= 1e-13


def test_repeat_runs_identical(dev, isw, grid4):
    """Two runs from the same state are bit-identical (no atomics, fixed summation order)."""
    a = run_stack(isw, grid4, golden('ocean2_n4'), dev, 3)
    b = run_stack(isw, grid4, golden('ocean2_n4'), dev, 3)
    for x, y in zip(a[1:4], b[1:4]):
        assert torch.equal(x, y)


def test_fp64_branches_on_a_mixed_grid(dev, isw, grid4):
    """Walls, the shelf and air layers asked of the mixed form step in the FP64 form (as the reference's mixed build
    keeps its air kernels in FP64): the object reports it, and its steps equal the FP64 grid's bit for bit."""
    from isw._lib import ISW_FP64
    gpu, layers, _ = isw
    gpu.set_precision('mixed')
    try:
        dgm = gpu.DeviceGrid(grid4)
    finally:
        gpu.set_precision('double')
    dgd = gpu.DeviceGrid(grid4)
    z = golden('outcrop_n4')
    for kw in (dict(wall=np.ones(dgm.E)), dict(shelf=50.0)):
        cores = [layers.Layers(dg, 2, b=z['b'], gprime=[0.02], stress=[0.0, 2.5e-4], nu4=float(z['nu4']), floor=1.0, **kw)
                 for dg in (dgm, dgd)]
        assert cores[0].precision == ISW_FP64
        states = [(T(z['h0'], dev), T(z['u0'], dev)) for _ in cores]
        for core, (h, u) in zip(cores, states):
            for _ in range(3):
                core.step(h, u, float(z['dt']), int(z['nfast']))
        torch.cuda.synchronize()
        assert torch.equal(states[0][0], states[1][0]) and torch.equal(states[0][1], states[1][1])
    air = layers.Layers(dgm, 2, gprime=[0.0], air={'cp': 1004.6})
    assert air.precision == ISW_FP64


def test_bad_arguments_rejected(dev, isw, grid4):
    gpu, layers, _ = isw
    dg = gpu.DeviceGrid(grid4)
    core = layers.Layers(dg, 1)
    h = torch.zeros(1, dg.N, dtype=torch.float64, device=dev)
    u = torch.zeros(1, dg.E, dtype=torch.float64, device=dev)
    with pytest.raises(ValueError):
        core.step(h[:, :10], u, 900.0, 2)
    with pytest.raises(TypeError):
        core.step(h.float(), u, 900.0, 2)
    with pytest.raises(ValueError):
        core.step(h, u, -1.0, 2)


def test_air_layers_golden(dev, isw, grid4):
    """Air layers (h = mass per area, theta per layer: the reference's air branch) from the reference's aquaplanet start,
    with surface drag, nabla^4, interfacial stress and its heating: the fast-mode coefficient's sub-step count equals
    the reference's, and h, u, theta and Fm after 1 and 12 steps equal the reference's to 1e-12 relative (the branch
    calls pow, whose last bit may differ between the host's libm and CUDA's)."""
    from isw import grid as G
    gpu, layers, _ = isw
    z = golden('airtheta_n4')
    dg = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616))
    core = layers.Layers(dg, 3, b=z['b'], gprime=[0.0, 0.0], stress=list(z['stress']), nu4=float(z['nu4']),
                         floor=float(z['floor']), vmix=float(z['vmix']),
                         air=dict(t_ref=288.0, cp=float(z['cp']), kappa=float(z['kappa']), rd=float(z['rd'])))
    h, u, theta = T(z['h0'], dev), T(z['u0'], dev), T(z['theta0'], dev)
    Fm = torch.zeros_like(u)
    dt, nfast = float(z['dt']), int(z['nfast'])
    core.update_gfast(h, theta)
    assert core.substeps(h, dt) == int(z['substeps'])
    worst = 0.0
    for s in range(1, 13):
        core.step(h, u, dt, nfast, Fm, theta=theta)
        if s in (1, 12):
            torch.cuda.synchronize()
            sfx = '1' if s == 1 else ''
            for name, x in (('h', h), ('u', u), ('theta', theta), ('Fm', Fm)):
                e = rel(x.cpu().numpy(), z[name + sfx])
                worst = max(worst, e)
                assert e <= REL, (s, name, e)
    with pytest.raises(ValueError):
        core.step(h, u, dt, nfast, Fm)                      # air layers need theta


def test_world_vmix_heat_call_golden(dev, isw, grid4):
    """The world's own launch of the layers' heating kernel after the sea coupling (reference world.py:317-318:
    core.k['vmix_heat'](*grid_dims(N), (N, L, h, sea.diss, g.cellEdge, g.le, g.de, g.areaCell, grav, core.cpa,
    core.kap, P0, theta))), made here exactly so with this core's Layers and DeviceGrid, against the reference kernel's
    own result: theta after two calls to 1e-12 relative (and its increments to 1e-10; the kernel calls pow, whose last
    bit may differ between the host's libm and CUDA's)."""
    from isw import grid as G
    gpu, layers, _ = isw
    z = golden('vmixheat_n4')
    g = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616))
    core = layers.Layers(g, 3, gprime=[0.0, 0.0], floor=10.0, air=dict(t_ref=288.0), vmix=5e-3)
    assert 'vmix_heat' in core.k and core.cpa == float(z['cp']) and core.kap == float(z['kappa'])
    h, diss, theta = T(z['h'], dev), T(z['diss'], dev), T(z['theta0'], dev)
    i32, R = np.int32, np.float64
    grid_dims = ((g.N + 255) // 256, 1), (256,)
    for call in (1, 2):
        core.k['vmix_heat'](*grid_dims, (i32(g.N), i32(3), h, diss, g.cellEdge, g.le, g.de, g.areaCell, R(z['grav']),
                                         R(core.cpa), R(core.kap), R(z['p0']), theta))
        torch.cuda.synchronize()
        got = theta.cpu().numpy()
        assert rel(got, z[f'theta{call}']) <= REL, call
        want_inc = z[f'theta{call}'] - (z['theta0'] if call == 1 else z['theta1'])
        prev = z['theta0'] if call == 1 else z['theta1']
        assert np.max(np.abs((got - prev) - want_inc)) <= 1e-10 * np.max(np.abs(want_inc))
        theta = T(z[f'theta{call}'], dev)
    with pytest.raises(ValueError):
        core.k['vmix_heat'](*grid_dims, (i32(g.N), i32(2), h, diss, g.cellEdge, g.le, g.de, g.areaCell, R(9.8), R(1004.0),
                                         R(0.28), R(1e5), theta))
    with pytest.raises(KeyError):
        core.k['lay_slow']


def test_wall_mask(dev, isw, grid4):
    """Layers.mask (reference layers.py:94-97, kernel lay_mask) zeroes the wall edges of the first rows of an edge
    field and leaves every other value; a Layers without walls leaves the field unchanged."""
    from isw import grid as G
    gpu, layers, _ = isw
    g = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616))
    wall = (np.arange(g.E) % 7 != 3).astype(np.float64)
    core = layers.Layers(g, 2, gprime=[0.02], wall=wall)
    a = torch.arange(3 * g.E, dtype=torch.float64, device=dev).reshape(3, g.E) + 1.0
    want = a.cpu().numpy().copy()
    want[:2, wall == 0] = 0
    core.mask(a[:2], 2)
    core.k['lay_mask'](((g.E + 255) // 256, 1), (256,), (np.int32(g.E), np.int32(2), core.wall, a[:2]))
    assert np.array_equal(a.cpu().numpy(), want)
    plain = layers.Layers(g, 2, gprime=[0.02])
    b = torch.ones(2, g.E, dtype=torch.float64, device=dev)
    plain.mask(b, 2)
    assert bool((b == 1).all())


def test_exchange_golden(dev, isw, grid4):
    """The between-step exchange hook (Layers.exchange) after one step, against the reference's own: Boussinesq layers
    with seeded thickness moves, plain and sequential (h, u, M and the tracer); air layers with the momentum mixing's
    heat, the step's nabla^4 loss and a nearly empty layer taking its neighbours' wind (h, u, M, tracer, theta). To
    1e-12 relative (the steps before call exp and pow)."""
    from isw import grid as G
    gpu, layers, _ = isw
    z = golden('exchange_n4')
    dg = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616))
    A = T(dg.host.areaCell, dev)
    core = layers.Layers(dg, 3, b=z['b_b'], gprime=list(z['b_gprime']), stress=list(z['b_stress']), nu4=float(z['b_nu4']),
                         floor=float(z['b_floor']), vmix=float(z['b_vmix']))
    h0, u0 = T(z['b_h0'], dev), T(z['b_u0'], dev)
    core.step(h0, u0, float(z['b_dt']), 20)
    for tag, seq in (('plain', False), ('seq', True)):
        h, u = h0.clone(), u0.clone()
        M = (h * A[None]).contiguous()
        psi = T(z['b_psi0'], dev)
        core.exchange(T(z['b_wx'], dev), h, u, M, psi, seq=seq)
        torch.cuda.synchronize()
        for name, x in (('h', h), ('u', u), ('M', M), ('psi', psi)):
            e = rel(x.cpu().numpy(), z[f'b_{tag}_{name}'])
            assert e <= REL, (tag, name, e)
    core = layers.Layers(dg, 3, b=np.zeros(dg.N), gprime=[0.0, 0.0], stress=[0.0, 0.0, float(z['a_drag'])],
                         nu4=float(z['a_nu4']), floor=10.0, thin_wind=100.0,
                         air=dict(t_ref=288.0, cp=float(z['a_cp']), kappa=float(z['a_kappa']), rd=float(z['a_rd'])))
    h, u, theta = T(z['a_h0'], dev), T(z['a_u0'], dev), T(z['a_theta0'], dev)
    core.update_gfast(h, theta)
    core.step(h, u, 1800.0, int(z['a_nfast']), theta=theta)
    M = (h * A[None]).contiguous()
    psi = T(z['a_psi0'], dev)
    core.exchange(T(z['a_wx'], dev), h, u, M, psi, theta=theta)
    torch.cuda.synchronize()
    for name, x in (('h', h), ('u', u), ('M', M), ('psi', psi), ('theta', theta)):
        e = rel(x.cpu().numpy(), z[f'a_{name}'])
        assert e <= REL, ('air', name, e)


def test_exchange_bit_exact(dev, isw, grid4):
    """The exchange hook alone, bit for bit against the reference's own xch_cell / xch_edge / lay_mask (built for the
    host in oracle/_ref) on seeded states: 2, 3 and 5 Boussinesq layers, moves of both signs and zero, all at once and
    in flow order, with thin walls; air layers with a nearly empty layer taking its neighbours' wind (h, u, M, psi bit
    for bit; theta, which goes through pow, to 1e-14)."""
    from oracle import refkernels
    if not refkernels.available():
        pytest.skip('oracle/_ref not built')
    from isw import grid as G
    gpu, layers, _ = isw
    K = refkernels.RefKernels()
    g = G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616)
    dg = gpu.DeviceGrid(g)
    N, E = g.N, g.E
    rng = np.random.default_rng(11)
    i32, f64 = np.int32, np.float64
    wall = (rng.random(E) > 0.05).astype(f64)

    def ref(L, h, u, M, psi, wx, seq, hthin=0.0, floor=1.0, theta=None, cp=1004.6, kap=287.04 / 1004.6, mask=None):
        h, u, M, psi = h.copy(), u.copy(), M.copy(), psi.copy()
        hold = h.copy()
        diss = np.zeros(E)
        K.launch('xch_cell', ((N + 255) // 256,), (256,), (i32(N), i32(L), wx, g.areaCell, h, M, psi, i32(seq)))
        K.launch('xch_edge', ((E + 255) // 256,), (256,), (i32(N), i32(E), i32(L), wx, hold, g.eI, g.eJ, u,
                                                           diss if theta is not None else 0, 0, f64(0.0), f64(hthin), f64(floor)))
        if mask is not None:
            K.launch('lay_mask', ((E + 255) // 256,), (256,), (i32(E), i32(L), mask, u))
        if theta is not None:
            theta = theta.copy()
            K.launch('vmix_heat', ((N + 255) // 256,), (256,), (i32(N), i32(L), h, diss, g.cellEdge, g.le, g.de, g.areaCell,
                                                               f64(9.80616), f64(cp), f64(kap), f64(1.0e5), theta))
        return h, u, M, psi, theta

    for L, seq, walls in ((2, 0, False), (3, 0, True), (3, 1, True), (5, 1, False), (5, 0, False)):
        h = 50.0 + 1000.0 * rng.random((L, N))
        u = 20.0 * rng.standard_normal((L, E))
        psi = rng.random((L, N))
        M = h * g.areaCell[None]
        wx = 10.0 * rng.standard_normal((L - 1, N))
        wx[rng.random((L - 1, N)) < 0.2] = 0.0
        core = layers.Layers(dg, L, gprime=[0.01] * (L - 1), wall=wall if walls else None)
        want = ref(L, h, u, M, psi, np.ascontiguousarray(wx), seq, mask=wall if walls else None)
        got = [T(a, dev) for a in (h, u, M, psi)]
        core.exchange(T(wx, dev), *got, seq=bool(seq))
        torch.cuda.synchronize()
        for name, x, w in zip('h u M psi'.split(), got, want):
            assert np.array_equal(x.cpu().numpy(), w), (L, seq, name, rel(x.cpu().numpy(), w))

    L = 3                                   # air: mass per area, a nearly empty middle layer in a quarter of the cells
    h = 2000.0 + 3000.0 * rng.random((L, N))
    h[1, rng.random(N) < 0.25] = 12.0 + 50.0 * rng.random()
    u = 15.0 * rng.standard_normal((L, E))
    psi, theta = rng.random((L, N)), 250.0 + 60.0 * rng.random((L, N))
    M = h * g.areaCell[None]
    wx = 3.0 * rng.standard_normal((L - 1, N))
    core = layers.Layers(dg, L, gprime=[0.0, 0.0], floor=10.0, thin_wind=100.0,
                         air=dict(t_ref=288.0, cp=1004.6, kappa=287.04 / 1004.6, rd=287.04))
    want = ref(L, h, u, M, psi, np.ascontiguousarray(wx), 0, hthin=100.0, floor=10.0, theta=theta)
    got = [T(a, dev) for a in (h, u, M, psi, theta)]
    core.exchange(T(wx, dev), *got[:4], theta=got[4])
    torch.cuda.synchronize()
    for name, x, w in zip('h u M psi'.split(), got, want):
        assert np.array_equal(x.cpu().numpy(), w), ('air', name, rel(x.cpu().numpy(), w))
    assert rel(got[4].cpu().numpy(), want[4]) <= 1e-14


def test_exchange_golden_after_batched_step(dev, isw, grid4):
    """The exchange hook on layers that step in a batch (the ocean's between-step moves, ocean.py:159 and :245): after
    one batched step, exchange equals the reference's golden vectors to 1e-12 (the step's stress calls exp)."""
    from isw import grid as G
    from isw.batch import Batch
    gpu, layers, _ = isw
    z = golden('exchange_n4')
    dg = gpu.DeviceGrid(G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616))
    A = T(dg.host.areaCell, dev)
    core = layers.Layers(dg, 3, b=z['b_b'], gprime=list(z['b_gprime']), stress=list(z['b_stress']), nu4=float(z['b_nu4']),
                         floor=float(z['b_floor']), vmix=float(z['b_vmix']))
    h0, u0 = T(z['b_h0'], dev), T(z['b_u0'], dev)
    batch = Batch(0)
    batch.add(core, h0, u0, torch.zeros_like(u0), dt=float(z['b_dt']), nfast=20)
    batch.step()
    torch.cuda.synchronize()
    for tag, seq in (('plain', False), ('seq', True)):
        h, u = h0.clone(), u0.clone()
        M = (h * A[None]).contiguous()
        psi = T(z['b_psi0'], dev)
        core.exchange(T(z['b_wx'], dev), h, u, M, psi, seq=seq)
        torch.cuda.synchronize()
        for name, x in (('h', h), ('u', u), ('M', M), ('psi', psi)):
            e = rel(x.cpu().numpy(), z[f'b_{tag}_{name}'])
            assert e <= REL, (tag, name, e)


def test_option_branches_golden(dev, isw, grid4):
    """Every option branch of Boussinesq layers at once on the reference's outcrop case (walls, the shelf with its bed
    flags, per-cell buoyancy, a tide potential, the bottom's quadratic and internal-tide drag), set as the reference's
    callers set them: h, u, Fm after 1 and 12 steps to 1e-12 of the reference's (its stress term calls exp), call by
    call and through a batch (beside a plain stack, with the grid-wide sub-steps split and persistent), the
    batched run equal to the call-by-call one bit for bit."""
    gpu, layers, _ = isw
    from isw.batch import Batch
    z = golden('options_n4')
    dg = gpu.DeviceGrid(grid4)
    sig, tide, cbot = T(z['sig'], dev), T(z['tide'], dev), T(z['cbot'], dev)
    dt, nfast = float(z['dt']), int(z['nfast'])

    def options_core():
        core = layers.Layers(dg, 2, b=z['b'], gprime=[0.02], stress=[0.0, 2.5e-4], nu4=float(z['nu4']), floor=1.0,
                             wall=z['wall'], shelf=50.0, shelf_bed=True)
        core.sig, core.zm = sig, torch.zeros_like(sig)
        core.tide = tide
        core.cd_bot = 2.5e-3
        core.cbot = cbot
        return core
    core = options_core()
    h, u = T(z['h0'], dev), T(z['u0'], dev)
    Fm = torch.zeros_like(u)
    assert core.substeps(h, dt) * 1.2 <= nfast
    for s in range(1, 13):
        core.step(h, u, dt, nfast, Fm)
        if s in (1, 12):
            torch.cuda.synchronize()
            sfx = '1' if s == 1 else ''
            for name, x in (('h', h), ('u', u), ('Fm', Fm)):
                e = rel(x.cpu().numpy(), z[name + sfx])
                assert e <= REL, (s, name, e)
    w2 = golden('w2_n4')
    for grid in ('split', 'persistent'):
        bcore = options_core()
        hb, ub = T(z['h0'], dev), T(z['u0'], dev)
        Fb = torch.zeros_like(ub)
        plain = layers.Layers(dg, 1, b=w2['b'])
        hp, up = T(w2['h0'], dev), T(w2['u0'], dev)
        batch = Batch(0)
        batch.config(grid=grid)
        batch.add(bcore, hb, ub, Fb, dt=dt, nfast=nfast)
        batch.add(plain, hp, up, torch.zeros_like(up), dt=float(w2['dt']), nfast=int(w2['nfast']))
        for _ in range(12):
            batch.step()
        torch.cuda.synchronize()
        assert batch.status() == 0
        assert torch.equal(hb, h) and torch.equal(ub, u) and torch.equal(Fb, Fm), grid
