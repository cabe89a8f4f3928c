"""The batched persistent step (isw.batch.Batch over the C ABI): each stack's result is bit-identical to stepping it
alone, across stacks of different grids and layer counts in one launch; the golden vectors hold through it; and a
grid barrier whose wait runs out reports ISW_ETIMEOUT to the host and leaves the context usable."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def dev():
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from isw import gpu
    gpu.set_precision('double')
    return torch.device('cuda:0')


def T(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)


def make_stack(dg, z, dev):
    from isw.layers import Layers
    from isw.transport import Transport
    L = int(z['L'])
    core = Layers(dg, L, b=z['b'], gprime=list(z['gprime']), stress=list(z['stress']), nu4=float(z['nu4']),
                  floor=float(z['floor']), vmix=float(z['vmix']), batched=False)   # call by call: the per-call kernels
    tr = Transport(dg, layers=L, tracers=3)
    st = dict(core=core, tr=tr, h=T(z['h0'], dev), u=T(z['u0'], dev))
    st['M'] = T(z['h0'] * dg.host.areaCell[None], dev)
    st['M1'] = torch.zeros_like(st['M'])
    st['Fm'] = torch.zeros_like(st['u'])
    st['trc'] = [T(z[f'tr{k}_0'], dev) for k in range(3)]
    return st


def percall(st, dt, nfast, steps):
    for _ in range(steps):
        st['core'].step(st['h'], st['u'], dt, nfast, st['Fm'])
        st['tr'].mass_after(st['M'], st['Fm'], st['M1'])
        st['tr'].step_many(st['M'], st['M1'], st['Fm'], st['trc'], order=3)
        st['M'].copy_(st['M1'])


def fields(st):
    return [st['h'], st['u'], st['M'], st['Fm']] + st['trc']


def test_batch_matches_percall_and_golden(dev, grid4):
    """Air and ocean stacks in one launch per step: equal to the call-by-call path bit for bit, and to the reference's
    golden vectors to 1e-12 (bit for bit where no exp() is involved)."""
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    dg = DeviceGrid(G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616))
    zs = [golden('air3_n4'), golden('ocean2_n4')]
    a = [make_stack(dg, z, dev) for z in zs]
    b = [make_stack(dg, z, dev) for z in zs]
    batch = Batch(0)
    for st, z in zip(b, zs):
        batch.add(st['core'], st['h'], st['u'], st['Fm'], tr=st['tr'], M=st['M'], M1=st['M1'], tracers=st['trc'],
                  dt=float(z['dt']), nfast=int(z['nfast']))
    for st, z in zip(a, zs):
        percall(st, float(z['dt']), int(z['nfast']), 6)
    for _ in range(6):
        batch.step()
    torch.cuda.synchronize()
    assert batch.status() == 0
    for sa, sb, z in zip(a, b, zs):
        for x, y in zip(fields(sa), fields(sb)):
            assert torch.equal(x, y)
        for name, x in (('h', sb['h']), ('u', sb['u']), ('M', sb['M'])):
            ref = z[name]
            assert float(np.max(np.abs(x.cpu().numpy() - ref)) / np.max(np.abs(ref))) <= 1e-12, name


def test_batch_w2_bit_exact(dev, grid4):
    """Williamson 2 through the batch (one layer, no transport): 480 steps equal the reference's bit for bit."""
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.layers import Layers
    z = golden('w2_n4')
    dg = DeviceGrid(G.for_planet(grid4, 6.371e6, float(z['omega']), 9.80616))
    core = Layers(dg, 1, b=z['b'])
    h, u = T(z['h0'], dev), T(z['u0'], dev)
    Fm = torch.zeros_like(u)
    batch = Batch(0)
    batch.add(core, h, u, Fm, dt=float(z['dt']), nfast=int(z['nfast']))
    for s in range(1, 481):
        batch.step()
        if s in (1, 96, 480):
            torch.cuda.synchronize()
            assert np.array_equal(h.cpu().numpy(), z[f'h{s}']) and np.array_equal(u.cpu().numpy(), z[f'u{s}']), s


def test_batch_mixed_levels_equal_alone(dev, grid4):
    """Members on level 3 and level 4 grids share one launch; each equals its own run alone, bit for bit."""
    from isw import cases
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    dg4 = DeviceGrid(planet_grid(grid4))
    dg3 = DeviceGrid(planet_grid(G.build(3, device='cpu')))
    batch = Batch(0)
    mixed = [Member(dg3, 5, nfast=20, batch=batch), Member(dg4, 6, nfast=20, batch=batch)]
    alone = [Member(dg3, 5, nfast=20), Member(dg4, 6, nfast=20)]
    for _ in range(4):
        batch.step()
        for m in alone:
            m.step()
    torch.cuda.synchronize()
    for mb, ma in zip(mixed, alone):
        for x, y in zip(mb.state(), ma.state()):
            assert torch.equal(x, y)


@pytest.mark.parametrize('levels', [{3: ('untiled', 0, 0), 4: ('packed', 256, 3)}, {3: ('packed', 128, 2), 4: ('untiled', 0, 0)}])
def test_batch_layout_per_level_equals_alone(dev, grid4, levels):
    """A layout per grid level in one batch (one level's stacks in packed tiles of their own size and interval, the
    other's grid-wide): each member equals its own run alone, bit for bit, and still does under the configuration the
    autotuner (with its per-level pass) leaves."""
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    dg4 = DeviceGrid(planet_grid(grid4))
    dg3 = DeviceGrid(planet_grid(G.build(3, device='cpu')))
    batch = Batch(0)
    mixed = [Member(dg3, 5, nfast=20, batch=batch), Member(dg4, 6, nfast=20, batch=batch)]
    alone = [Member(dg3, 5, nfast=20), Member(dg4, 6, nfast=20)]
    batch.config(tiles=True, layout='packed', levels=levels)
    info = batch.info()
    assert info['tiles'] > 0 and info['groups'] >= 1
    for _ in range(4):
        batch.step()
        for m in alone:
            m.step()
    torch.cuda.synchronize()
    for mb, ma in zip(mixed, alone):
        for x, y in zip(mb.state(), ma.state()):
            assert torch.equal(x, y)
    best, times = batch.autotune(steps=1)
    batch.step()
    for m in alone:
        m.step()
    torch.cuda.synchronize()
    for mb, ma in zip(mixed, alone):
        for x, y in zip(mb.state(), ma.state()):
            assert torch.equal(x, y)


def test_barrier_timeout_refuses_then_recovers(dev, grid4):
    """A block that never arrives at a grid barrier: the others' bounded waits run out and the host reads ISW_ETIMEOUT.
    While the status is set the batch refuses to step (ISW_ETIMEOUT, nothing launched), so a caller that never polls
    cannot step on a half-updated state. Once reset, the SAME batch steps again and equals an untouched run of the same
    member bit for bit (the timed-out launch wrote only the fast loop's scratch, which every step rebuilds from h, u)."""
    from isw._lib import ISW_ETIMEOUT, IswError
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    dg = DeviceGrid(planet_grid(grid4))
    batch = Batch(0)
    a = Member(dg, 4, nfast=20, batch=batch)
    b = Member(dg, 4, nfast=20)
    batch.fault_test(timeout_s=0.05)
    torch.cuda.synchronize()
    with pytest.raises(IswError) as err:
        batch.step()
    assert err.value.status == ISW_ETIMEOUT
    assert batch.status() == ISW_ETIMEOUT
    assert batch.status(reset=True) == ISW_ETIMEOUT
    assert batch.status() == 0
    for _ in range(2):
        batch.step()
        b.step()
    torch.cuda.synchronize()
    assert batch.status() == 0
    for x, y in zip(a.state(), b.state()):
        assert torch.equal(x, y)


@pytest.mark.parametrize('precision', ['double', 'mixed'])
def test_nonfinite_thickness_reported_and_refused(dev, grid4, precision):
    """A NaN written into one thickness from the host: the step that meets it records ISW_ENOTFINITE (checked for every
    cell and layer at the step's end) and the batch refuses further steps until the status is reset; after the state is
    restored and the status reset, the same batch steps on equal to an untouched run bit for bit. The Layers path
    (one-stack batch) refuses the same way and reports through Layers.status."""
    from isw import gpu
    from isw._lib import ISW_ENOTFINITE, IswError
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    gpu.set_precision(precision)
    try:
        dg = DeviceGrid(planet_grid(grid4))
        batch, other = Batch(0), Batch(0)
        a = Member(dg, 5, nfast=20, batch=batch)
        b = Member(dg, 5, nfast=20, batch=other)         # the untouched run: the same batched path
        c = Member(dg, 5, nfast=20)
    finally:
        gpu.set_precision('double')
    saved = [x.clone() for x in a.state()]
    a.stacks[1].h[1, 17] = float('nan')
    batch.step()
    torch.cuda.synchronize()
    assert batch.status() == ISW_ENOTFINITE
    with pytest.raises(IswError) as err:
        batch.step()
    assert err.value.status == ISW_ENOTFINITE
    for x, y in zip(a.state(), saved):
        x.copy_(y)
    assert batch.status(reset=True) == ISW_ENOTFINITE
    for _ in range(2):
        batch.step()
        b.step()
    torch.cuda.synchronize()
    assert batch.status() == 0
    for x, y in zip(a.state(), b.state()):
        assert torch.equal(x, y)
    s = c.stacks[0]
    s.h[0, 5] = float('inf')
    s.step()
    torch.cuda.synchronize()
    assert s.core.status() == ISW_ENOTFINITE
    with pytest.raises(IswError):
        s.step()
    assert s.core.status(reset=True) == ISW_ENOTFINITE and s.core.status() == 0


@pytest.mark.parametrize('k', [1, 2, 3, 4, 7, 8])
def test_tiled_fast_loop_equals_grid_wide(dev, grid4, k):
    """The barotropic sub-steps in shared-memory tiles (exchanging every k sub-steps) give the grid-wide passes' result
    bit for bit, and so does the call-by-call path."""
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    dg = DeviceGrid(planet_grid(grid4))
    tiled, flat = Batch(0), Batch(0)
    tiled.config(tiles=True, tile_k=k)
    flat.config(tiles=False)
    a, b, c = Member(dg, 9, batch=tiled), Member(dg, 9, batch=flat), Member(dg, 9)
    info = tiled.info()
    assert info['tiles'] > 0 and 1 <= info['tile_k'] <= k
    for _ in range(3):
        tiled.step()
        flat.step()
        c.step()
    torch.cuda.synchronize()
    assert tiled.status() == 0 and flat.status() == 0
    for x, y, z in zip(a.state(), b.state(), c.state()):
        assert torch.equal(x, y) and torch.equal(x, z)


@pytest.mark.parametrize('precision', ['double', 'mixed'])
def test_grid_wide_forms_equal(dev, grid4, precision):
    """The grid-wide sub-steps as two launches each (over wide chunks, several items a thread) give the persistent
    loop's result (item by item) bit for bit: members of different sub-step counts in one batch (nfast 20, 7 and 2, the
    last with stages of one sub-step), and a grid-wide level beside a tiled one (the layer fluxes then formed in phase
    C)."""
    from isw import gpu
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    gpu.set_precision(precision)
    try:
        dg4 = DeviceGrid(planet_grid(grid4))
        dg3 = DeviceGrid(planet_grid(G.build(3, device='cpu')))
        uneven, beside = {}, {}
        for grid in ('split', 'persistent'):
            bt = Batch(0)
            bt.config(tiles=False, grid=grid)
            uneven[grid] = (bt, [Member(dg4, 30, nfast=20, ntracers=2, batch=bt, fp64_kinds=()),
                                 Member(dg4, 31, nfast=7, ntracers=2, batch=bt, fp64_kinds=()),
                                 Member(dg4, 32, nfast=2, dt=60.0, ntracers=2, batch=bt, fp64_kinds=())])
            bt = Batch(0)
            bt.config(tiles=True, layout='packed', grid=grid, levels={3: ('packed', 128, 2), 4: ('untiled', 0, 0)})
            beside[grid] = (bt, [Member(dg3, 5, nfast=20, ntracers=2, batch=bt, fp64_kinds=()),
                                 Member(dg4, 6, nfast=20, ntracers=2, batch=bt, fp64_kinds=())])
    finally:
        gpu.set_precision('double')
    assert uneven['persistent'][0].info()['grid'] == 'persistent' and beside['split'][0].info()['tiles'] > 0
    for _ in range(3):
        for bt, _m in list(uneven.values()) + list(beside.values()):
            bt.step()
    torch.cuda.synchronize()
    for group in (uneven, beside):
        ref = group['split'][1]
        for grid, (bt, ms) in group.items():
            assert bt.status() == 0, grid
            for a, b in zip(ms, ref):
                for x, y in zip(a.state(), b.state()):
                    assert torch.equal(x, y), grid


def test_batch_of_both_forms(dev, grid4):
    """One batch holding FP64 and mixed stacks (each phase one kernel per form, the mixed stacks' fast loop in tiles, the
    FP64 stacks' as grid-wide sub-steps): every FP64 stack equals the same stack in an FP64-only batch bit for bit, and
    every mixed stack equals the same stack in a mixed-only batch bit for bit."""
    from isw import gpu
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    dg = DeviceGrid(planet_grid(grid4))
    gpu.set_precision('mixed')
    try:
        dgm = DeviceGrid(planet_grid(grid4))
    finally:
        gpu.set_precision('double')
    both, only64, onlym = Batch(0), Batch(0), Batch(0)
    a = [Member(dgm, 60, ntracers=2, batch=both, fp64_kinds=('ocean',)), Member(dg, 61, ntracers=2, batch=both)]
    b = [Member(dg, 60, ntracers=2, batch=only64, kinds=('ocean',)), Member(dg, 61, ntracers=2, batch=only64)]
    c = Member(dgm, 60, ntracers=2, batch=onlym, kinds=('air',), fp64_kinds=())
    assert [s.core.precision for s in a[0].stacks] == [1, 0]
    info = both.info()
    assert info['tiles'] > 0, info
    for _ in range(4):
        for bt in (both, only64, onlym):
            bt.step()
    torch.cuda.synchronize()
    for bt in (both, only64, onlym):
        assert bt.status() == 0
    pairs = list(zip(a[0].stacks[1].state(), b[0].stacks[0].state())) + list(zip(a[1].state(), b[1].state()))
    pairs += list(zip(a[0].stacks[0].state(), c.stacks[0].state()))
    for x, y in pairs:
        assert torch.equal(x, y)


@pytest.mark.parametrize('precision', ['double', 'mixed'])
def test_packed_groups_equal_shared(dev, grid4, precision):
    """Eight members in the packed layout (tiles of about 64 owned cells, more tiles than one cooperative launch holds,
    so the fast loop runs as several launches per stage) give the shared layout's result bit for bit; in FP64 also the
    grid-wide passes' result."""
    from isw import gpu
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    gpu.set_precision(precision)
    try:
        dg = DeviceGrid(planet_grid(grid4))
        packed, shared, flat = Batch(0), Batch(0), Batch(0)
        packed.config(tiles=True, tile_k=4, layout='packed', tile_cells=64, blocks_per_sm=2)
        shared.config(tiles=True, tile_k=4, layout='shared')
        flat.config(tiles=False)
        ms = [[Member(dg, 20 + i, ntracers=2, batch=bt, fp64_kinds=()) for i in range(8)] for bt in (packed, shared, flat)]
    finally:
        gpu.set_precision('double')
    info = packed.info()
    assert info['groups'] >= 2 and info['tiles'] > 296, info
    for _ in range(3):
        for bt in (packed, shared, flat):
            bt.step()
    torch.cuda.synchronize()
    for bt in (packed, shared, flat):
        assert bt.status() == 0
    for a, b, c in zip(*ms):
        for x, y, z in zip(a.state(), b.state(), c.state()):
            assert torch.equal(x, y)
            if precision == 'double':
                assert torch.equal(x, z)
            else:
                assert float(torch.max(torch.abs(x - z)) / torch.max(torch.abs(z))) <= 1e-5


def test_autotune_keeps_state(dev, grid4):
    """The autotuner times candidate layouts on the live batch and restores every registered array: the stepped result
    afterwards equals an untuned batch's bit for bit."""
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    dg = DeviceGrid(planet_grid(grid4))
    tuned, plain = Batch(0), Batch(0)
    a, b = Member(dg, 5, batch=tuned), Member(dg, 5, batch=plain)
    best, times = tuned.autotune(steps=2)
    assert best in [dict(k) for k in times] and len(times) >= 2
    for _ in range(3):
        tuned.step()
        plain.step()
    torch.cuda.synchronize()
    for x, y in zip(a.state(), b.state()):
        assert torch.equal(x, y)


@pytest.mark.parametrize('precision', ['double', 'mixed'])
def test_pipelined_equals_plain(dev, grid4, precision):
    """A pipelined batch (each step's dynamics beside the previous step's transport) gives, after flush(), the plain
    order's h, u, M, Fm and tracers bit for bit, for an odd and an even number of steps; a stack added midway is
    flushed in first and the result still matches."""
    from isw import gpu
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    gpu.set_precision(precision)
    try:
        dg = DeviceGrid(planet_grid(grid4))
        for steps in (5, 6):
            plain, piped = Batch(0), Batch(0)
            piped.pipeline(True)
            a, b = Member(dg, 31, batch=plain), Member(dg, 31, batch=piped)
            for _ in range(steps):
                plain.step()
                piped.step()
            piped.flush()
            torch.cuda.synchronize()
            for sa, sb in zip(a.stacks, b.stacks):
                for x, y in zip(sa.state() + [sa.Fm], sb.state() + [sb.Fm]):
                    assert torch.equal(x, y), steps
        plain.step()
        piped.step()                                                      # a transport pending ...
        c, d = Member(dg, 32, batch=plain), Member(dg, 32, batch=piped)   # ... which adding a stack flushes first
        for _ in range(3):
            plain.step()
            piped.step()
        piped.flush()
        torch.cuda.synchronize()
        for x, y in zip(a.state() + c.state(), b.state() + d.state()):
            assert torch.equal(x, y)
    finally:
        gpu.set_precision('double')


def _air_world(dg, z, dev, batched_core=True):
    """Air layers from the reference's aquaplanet golden case with a tracer and theta moved by the transport (the
    reference's world tick moves theta with its tracers, world.py:291-301)."""
    from isw.layers import Layers
    from isw.transport import Transport
    L = int(z['h0'].shape[0])
    core = Layers(dg, L, b=z['b'], gprime=[0.0] * (L - 1), stress=list(z['stress']), nu4=float(z['nu4']),
                  floor=float(z['floor']), vmix=float(z['vmix']),
                  air=dict(t_ref=288.0, cp=float(z['cp']), kappa=float(z['kappa']), rd=float(z['rd'])))
    st = dict(core=core, tr=Transport(dg, layers=L, tracers=2), h=T(z['h0'], dev), u=T(z['u0'], dev),
              theta=T(z['theta0'], dev))
    st['M'] = (st['h'] * T(dg.host.areaCell, dev)[None]).contiguous()
    st['M1'] = torch.zeros_like(st['M'])
    st['Fm'] = torch.zeros_like(st['u'])
    st['trc'] = [T(np.stack([np.linspace(0.0, 1.0, dg.N)] * L), dev), st['theta']]
    core.update_gfast(st['h'], st['theta'])
    return st


@pytest.mark.parametrize('grid', ['split', 'persistent'])
def test_air_stack_in_batch_equals_per_call(dev, grid4, grid):
    """Air layers registered in a batch (isw_batch_add_air) beside a Boussinesq stack: 12 batched steps equal 12 ticks
    of Layers.step(theta=) + mass_after + step_many([psi, theta]) + M <- M1 call by call, bit for bit (h, u, M, Fm,
    the tracer and theta), with the grid-wide sub-steps as two launches each or as one persistent launch per stage;
    the Boussinesq stack equals its own call-by-call run."""
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    dg = DeviceGrid(G.for_planet(grid4, 6.371e6, 7.292e-5, 9.80616))
    za, zb = golden('airtheta_n4'), golden('air3_n4')
    dt, nfast = float(za['dt']), int(za['nfast'])
    ref = _air_world(dg, za, dev)
    for _ in range(12):
        ref['core'].step(ref['h'], ref['u'], dt, nfast, ref['Fm'], theta=ref['theta'])
        ref['tr'].mass_after(ref['M'], ref['Fm'], ref['M1'])
        ref['tr'].step_many(ref['M'], ref['M1'], ref['Fm'], ref['trc'], order=3)
        ref['M'].copy_(ref['M1'])
    bous_ref = make_stack(dg, zb, dev)
    percall(bous_ref, float(zb['dt']), int(zb['nfast']), 12)
    air = _air_world(dg, za, dev)
    bous = make_stack(dg, zb, dev)
    batch = Batch(0)
    batch.config(tiles=False, grid=grid)
    batch.add(air['core'], air['h'], air['u'], air['Fm'], tr=air['tr'], M=air['M'], M1=air['M1'], tracers=air['trc'],
              dt=dt, nfast=nfast, theta=air['theta'])
    batch.add(bous['core'], bous['h'], bous['u'], bous['Fm'], tr=bous['tr'], M=bous['M'], M1=bous['M1'],
              tracers=bous['trc'], dt=float(zb['dt']), nfast=int(zb['nfast']))
    for _ in range(12):
        batch.step()
    torch.cuda.synchronize()
    assert batch.status() == 0
    for x, y in zip(fields(air) + [air['theta']], fields(ref) + [ref['theta']]):
        assert torch.equal(x, y)
    for x, y in zip(fields(bous), fields(bous_ref)):
        assert torch.equal(x, y)
    with pytest.raises(ValueError):
        batch.add(air['core'], air['h'], air['u'], air['Fm'], dt=dt, nfast=nfast)        # air layers need theta


def test_autotune_two_level6_members(dev):
    """The autotuner's candidates include tilings that cannot be built for two level-6 members (a region too large for
    the tiles' 16-bit local ids); the planner leaves such stacks untiled instead of failing, and the tuned batch steps
    the members to the same state as untuned ones."""
    from isw import grid as G
    from isw.batch import Batch
    from isw.gpu import DeviceGrid
    from isw.workload import Member, planet_grid
    dg = DeviceGrid(planet_grid(G.build(6, device=0)))
    batch = Batch(0)
    tuned = [Member(dg, s, nfast=20, batch=batch) for s in (1, 2)]
    plain = Batch(0)
    plain.config(tiles=False)
    ref = [Member(dg, s, nfast=20, batch=plain) for s in (1, 2)]
    best, times = batch.autotune(steps=1)
    assert len(times) > 2
    for _ in range(2):
        batch.step()
        plain.step()
    torch.cuda.synchronize()
    assert batch.status() == 0
    for a, b in zip(tuned, ref):
        for x, y in zip(a.state(), b.state()):
            assert torch.equal(x, y)
