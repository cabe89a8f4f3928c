"""Generate the golden vectors in tests/golden/ by running the REFERENCE's own Python (``insilica.gpu``,
``insilica.layers``, ``insilica.transport``, ``insilica.grid``, ``insilica.cases``; unchanged, imported from the
reference checkout) on a NumPy-backed CuPy stand-in (``fakecupy.py``) whose kernels are the reference's own CUDA C
compiled for the host (``oracle/build_ref.py``), in the reference's FP64 form (``INSILICA_PRECISION=double``).

Needs the reference sources (``--ref``, else where ``oracle/refpath.py`` finds them) and ``oracle/_ref`` built. Run
from the repository root:

    python tests/golden/make_golden.py [--ref <reference checkout>] [--cache <grid cache directory>]

Fixtures written (compressed .npz; every array is stored with its SHA-256 too):
- grid_n4.npz    the reference's level-4 grid (Hilbert order), the arrays the step, the tables and the states use
- w2_n4.npz      Williamson 2, one layer, dt 900 s, Omega 7.292e-5: states after 1, 96 and 480 steps
- air3_n4.npz    three-layer air stack (terrain, nu4, interfacial stress, nfast 20, 3 FCT tracers): 6 steps
- ocean2_n4.npz  two-layer ocean stack (bottom and interfacial stress): 6 steps
- outcrop_n4.npz the reference's own 'outcrop' case (floor, stress, nu4) with the cosine-bell tracer: 24 steps
- bell_n4.npz    transport alone (solid-body flux): 20 steps of order 1 and of order 3
- dsum.npz       deterministic tree sums of fixed inputs
- airtheta_n4.npz the reference's air layers (h = mass per area, theta per layer; layers.py air branch) from its own
                 aquaplanet start (cases.aqua), surface drag, nabla^4, interfacial stress with its heating: 12 steps
- exchange_n4.npz the between-step exchange hook (Layers.exchange): Boussinesq layers after one step, seeded thickness
                 moves, plain and sequential; air layers after one step, with heating and the thin layers' wind
- options_n4.npz the option branches on the reference's outcrop case: thin walls, the shelf with its bed flags,
                 per-cell buoyancy (sig, zm), a tide potential, the bottom's quadratic and internal-tide drag: 12 steps
- vmixheat_n4.npz the world's call of the layers' heating kernel after the sea coupling (world.py:317-318:
                 core.k['vmix_heat'] with the sea's per-edge dissipation), on the aquaplanet's air layers: two calls

`--only NAME` writes one fixture (e.g. `--only airtheta`).
"""
import argparse
import hashlib
import math
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

GRID_KEYS = ('n', 'N', 'E', 'NV', 'eI', 'eJ', 'eKi', 'eKj', 'nbr', 'deg', 'cellEdge', 'cellEdgeAsc', 'cellSign', 'ev1', 'ev2',
             'vEdge', 'vEdgeSign', 'vCell', 'vSlot', 'eoeStart', 'eoe', 'cornerV', 'circ1', 'circ2', 'perm',
             'le', 'de', 'dist', 'edgeLen', 'areaCell', 'areaV', 'area', 'kite', 'w', 'fV', 'pos', 'lat', 'lon', 'xm', 'ne',
             'vPos', 'lloydIters')


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def save(name, d):
    out = {}
    for k, v in d.items():
        v = np.asarray(v)
        out[k] = v
        if v.dtype.kind in 'fiub' and v.ndim > 0:
            out[f'sha_{k}'] = np.asarray(sha(v))
    np.savez_compressed(HERE / name, **out)
    print(name, (HERE / name).stat().st_size, 'bytes')


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=None)
    ap.add_argument('--cache', default=None, help='the reference grid cache (default: a temporary directory)')
    ap.add_argument('--only', default=None)
    a = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    from oracle import refpath
    if a.ref is None:
        a.ref = refpath.reference_root()
        if a.ref is None:
            sys.exit('make_golden: reference checkout not found (pass --ref or set ISW_REFERENCE)')
    if a.cache is None:
        import tempfile
        a.cache = tempfile.mkdtemp(prefix='isw-grid-cache-')
    os.environ['INSILICA_PRECISION'] = 'double'
    os.environ['INSILICA_CACHE'] = a.cache
    sys.path.insert(0, str(HERE))
    sys.path.insert(0, str(Path(a.ref) / 'src'))
    sys.path.insert(0, str(ROOT / 'insilica-world-v2_b200'))
    import fakecupy
    fakecupy.install()
    cp = fakecupy
    from insilica import cases as rcases
    from insilica import grid as gridmod
    from insilica.gpu import DeviceGrid, dsum
    from insilica.layers import Layers
    from insilica.transport import Transport
    from isw import cases as mycases

    base = gridmod.get(4)
    g = gridmod.for_planet(base, 6.371e6, 7.292e-5, 9.80616)
    dg = DeviceGrid(g)
    if a.only == 'airtheta':
        save('airtheta_n4.npz', air_theta(cp, g, dg, Layers, rcases, mycases))
        return
    if a.only == 'options':
        save('options_n4.npz', options(cp, base, Layers, DeviceGrid, rcases, mycases))
        return
    if a.only == 'exchange':
        save('exchange_n4.npz', exchange(cp, g, dg, Layers, rcases, mycases))
        return
    if a.only == 'vmixheat':
        save('vmixheat_n4.npz', vmix_heat(cp, g, dg, Layers, rcases))
        return
    save('grid_n4.npz', {k: getattr(base, k) for k in GRID_KEYS})

    # ---- Williamson 2, one layer ----
    h0, b, u0 = rcases.initial_state(g, 'w2')
    core = Layers(dg, 1, b=b)
    h, u = cp.asarray(h0[None]), cp.asarray(u0[None])
    dt = 900.0
    sub = core.substeps(h, dt)
    nfast = int(math.ceil(1.2 * sub))
    d = dict(omega=7.292e-5, dt=dt, substeps=sub, nfast=nfast, h0=h0[None], u0=u0[None], b=b, energy0=core.energy(h, u))
    for s in range(1, 481):
        core.step(h, u, dt, nfast)
        if s in (1, 96, 480):
            d[f'h{s}'], d[f'u{s}'] = h.get(), u.get()
    d['energy480'] = core.energy(h, u)
    save('w2_n4.npz', d)

    # ---- the stacked-layer workloads (this project's synthetic states) at n = 4, 6 steps with transport ----
    def run_stack(kind, steps, dt, seed=7):
        s = mycases.stack_state(g, kind, seed)
        L = s['L']
        core = Layers(dg, L, b=s['b'], gprime=s['gprime'], stress=s['stress'], nu4=s['nu4'], floor=s['floor'], vmix=s['vmix'])
        tr = Transport(dg, layers=L, tracers=3)
        h, u = cp.asarray(s['h']), cp.asarray(s['u'])
        M = cp.asarray(s['h'] * g.areaCell[None])
        trc = [cp.asarray(t) for t in s['tracers']]
        Fm, M1 = cp.zeros((L, g.E)), cp.zeros((L, g.N))
        out = dict(kind=kind, seed=seed, L=L, dt=dt, nfast=20, h0=s['h'], u0=s['u'], b=s['b'], gprime=s['gprime'],
                   stress=s['stress'], nu4=s['nu4'], floor=s['floor'], vmix=s['vmix'], lap_max=core.lap_max(),
                   substeps=core.substeps(h, dt),
                   energy0=core.energy(h, u))
        for k, t in enumerate(s['tracers']):
            out[f'tr{k}_0'] = t
        for st in range(1, steps + 1):
            core.step(h, u, dt, 20, Fm)
            tr.mass_after(M, Fm, M1)
            tr.step_many(M, M1, Fm, trc, order=3)
            cp.copyto(M, M1)
            if st == 1:
                out['sha_h1'], out['sha_u1'] = sha(h), sha(u)
                out['sha_M1'] = sha(M)
                for k, t in enumerate(trc):
                    out[f'sha_tr{k}_1'] = sha(t)
        out.update(h=h.get(), u=u.get(), M=M.get(), Fm=Fm.get(), energy=core.energy(h, u))
        for k, t in enumerate(trc):
            out[f'tr{k}'] = t.get()
        return out

    save('air3_n4.npz', run_stack('air', 6, mycases.stack_dt(4)))
    save('ocean2_n4.npz', run_stack('ocean', 6, mycases.stack_dt(4)))

    # ---- the reference's own outcrop case (reference cases.py:174-182, PRESETS['outcrop']), with the bell tracer ----
    g0 = base
    dg0 = DeviceGrid(g0)
    ho, bo, uo = rcases.outcrop(g0)
    nu4 = mycases.visc4(g0, 0.5)
    core = Layers(dg0, 2, b=bo, gprime=[0.02], stress=[0.0, 2.5e-4], nu4=nu4, floor=1.0)
    tr = Transport(dg0, layers=2, tracers=4)
    h, u = cp.asarray(ho), cp.asarray(uo)
    dt = 3600.0
    nfast = int(math.ceil(1.2 * core.substeps(h, dt)))
    M = cp.asarray(ho * g0.areaCell[None])
    psi = cp.asarray(np.tile(rcases.cosine_bell(g0), (2, 1)))
    d = dict(dt=dt, nfast=nfast, nu4=nu4, h0=ho, u0=uo, b=bo, psi0=psi.get(), lap_max=core.lap_max())
    Fm, M1 = cp.zeros((2, g0.E)), cp.zeros((2, g0.N))
    lo = float(h.min())
    for st in range(1, 25):
        core.step(h, u, dt, nfast, Fm)
        tr.mass_after(M, Fm, M1)
        tr.step_many(M, M1, Fm, [psi], order=3)
        cp.copyto(M, M1)
        lo = min(lo, float(h.min()))
    d.update(h=h.get(), u=u.get(), M=M.get(), psi=psi.get(), Fm=Fm.get(), hmin=lo)
    save('outcrop_n4.npz', d)

    # ---- transport alone: the cosine bell in solid-body rotation (reference tests/test_accuracy.py:32-48) ----
    steps = 576
    dtb = 12 * 86400 / steps
    _, fm = mycases.solid_body_flux(g0, dtb)
    d = dict(dt=dtb, Fm=fm[None], psi0=rcases.cosine_bell(g0)[None], M0=g0.areaCell[None])
    for order in (1, 3):
        trb = Transport(dg0)
        psi = cp.asarray(d['psi0'])
        Mb, Mb1 = cp.asarray(d['M0']), cp.zeros((1, g0.N))
        Fmb = cp.asarray(d['Fm'])
        for _ in range(20):
            trb.mass_after(Mb, Fmb, Mb1)
            trb.step(Mb, Mb1, Fmb, psi, order)
            Mb, Mb1 = Mb1, Mb
        d[f'psi_o{order}'], d[f'M_o{order}'] = psi.get(), Mb.get()
    save('bell_n4.npz', d)

    # ---- deterministic sums (reference gpu.py:111-126, kernels/trisk.cu:61-81) ----
    d = {}
    for n in (1, 2, 255, 2048, 2049, 100003, 1 << 20):
        i = np.arange(n, dtype=np.int64)
        x = ((i * 7919) % 10007 - 5003) / 997.0
        y = ((i * 104729) % 65521) / 4093.0
        d[f'x_{n}'] = dsum(cp.asarray(x))
        d[f'xy_{n}'] = dsum(cp.asarray(x), cp.asarray(y))
    save('dsum.npz', d)
    save('airtheta_n4.npz', air_theta(cp, g, dg, Layers, rcases, mycases))
    save('exchange_n4.npz', exchange(cp, g, dg, Layers, rcases, mycases))
    save('options_n4.npz', options(cp, base, Layers, DeviceGrid, rcases, mycases))


def options(cp, g0, Layers, DeviceGrid, rcases, mycases):
    """The reference's outcrop case (two layers over a ridge that pierces the lower one) with every option branch on:
    5% of the edges walled (seeded), shelf 50 m with the bed flags, per-cell buoyancy sigma = (0, 0.02 (1 + 0.05 r)) for
    the fixed g', a tide potential 0.5 sin(2 lon) cos^2(lat) m^2/s^2, bottom quadratic drag 2.5e-3 and an internal-tide
    drag U(0, 1e-4) m/s per edge; 12 steps of 3600 s."""
    rng = np.random.default_rng(5)
    dg0 = DeviceGrid(g0)
    ho, bo, uo = rcases.outcrop(g0)
    nu4 = mycases.visc4(g0, 0.5)
    wall = np.where(rng.uniform(0, 1, g0.E) < 0.05, 0.0, 1.0)
    core = Layers(dg0, 2, b=bo, gprime=[0.02], stress=[0.0, 2.5e-4], nu4=nu4, floor=1.0, wall=wall, shelf=50.0,
                  shelf_bed=True)
    sig = np.stack([np.zeros(g0.N), 0.02 * (1 + 0.05 * rng.uniform(-1, 1, g0.N))])
    tide = 0.5 * np.sin(2 * g0.lon) * np.cos(g0.lat) ** 2
    cbot = rng.uniform(0.0, 1e-4, g0.E)
    core.sig, core.zm = cp.asarray(sig), cp.zeros((2, g0.N))
    core.tide = cp.asarray(tide)
    core.cd_bot = 2.5e-3
    core.cbot = cp.asarray(cbot)
    h, u = cp.asarray(ho), cp.asarray(uo)
    dt = 3600.0
    nfast = int(math.ceil(1.2 * core.substeps(h, dt)))
    Fm = cp.zeros((2, g0.E))
    d = dict(dt=dt, nfast=nfast, nu4=nu4, h0=ho, u0=uo, b=bo, wall=wall, sig=sig, tide=tide, cbot=cbot)
    for st in range(1, 13):
        core.step(h, u, dt, nfast, Fm)
        if st == 1:
            d.update(h1=h.get(), u1=u.get(), Fm1=Fm.get())
    d.update(h=h.get(), u=u.get(), Fm=Fm.get(), zm=core.zm.get())
    return d


def exchange(cp, g, dg, Layers, rcases, mycases):
    """Layers.exchange after one step: (1) the three-layer Boussinesq stack with seeded moves wx ~ U(-20, 20) m, plain
    and sequential, the demo tracer and masses; (2) the reference's air layers (aqua start, nabla^4, thin_wind 100 kg/m^2,
    one layer pressed near its floor in a band of cells) with wx ~ U(-300, 300) kg/m^2, heating theta."""
    rng = np.random.default_rng(11)
    out = {}
    s = mycases.stack_state(g, 'air', 7)
    core = Layers(dg, 3, b=s['b'], gprime=s['gprime'], stress=s['stress'], nu4=s['nu4'], floor=s['floor'], vmix=s['vmix'])
    h, u = cp.asarray(s['h']), cp.asarray(s['u'])
    core.step(h, u, mycases.stack_dt(4), 20)
    wx = rng.uniform(-20.0, 20.0, (2, g.N))
    psi0 = rng.uniform(0.0, 1.0, (3, g.N))
    out.update(b_h0=s['h'], b_u0=s['u'], b_b=s['b'], b_gprime=np.array(s['gprime']), b_stress=np.array(s['stress']),
               b_nu4=s['nu4'], b_floor=s['floor'], b_vmix=s['vmix'], b_dt=mycases.stack_dt(4), b_wx=wx, b_psi0=psi0)
    for seq in (False, True):
        hh, uu = h.copy(), u.copy()
        M = hh * cp.asarray(g.areaCell)[None]
        psi = cp.asarray(psi0)
        core.exchange(cp.asarray(wx), hh, uu, M, psi, seq=seq)
        tag = 'seq' if seq else 'plain'
        out.update({f'b_{tag}_h': hh.get(), f'b_{tag}_u': uu.get(), f'b_{tag}_M': M.get(), f'b_{tag}_psi': psi.get()})
    h0, b, u0, x = rcases.aqua(g)
    h0 = h0.copy()
    band = np.abs(g.lat - 0.3) < 0.1
    h0[2, band] = 60.0                                         # a nearly empty bottom layer in a band (thin_wind acts)
    theta0 = x['theta']
    nu4 = mycases.visc4(g, 15.0)
    core = Layers(dg, 3, b=b, gprime=[0.0, 0.0], stress=[0.0, 0.0, rcases.SURFACE_DRAG], nu4=nu4, floor=10.0,
                  air=dict(t_ref=288.0), thin_wind=100.0)
    h, u, theta = cp.asarray(h0), cp.asarray(u0), cp.asarray(theta0)
    core.update_gfast(h, theta)
    nfast = int(math.ceil(1.2 * core.substeps(h, 1800.0)))
    core.step(h, u, 1800.0, nfast, theta=theta)
    wx = rng.uniform(-300.0, 300.0, (2, g.N))
    wx[1, band] = np.minimum(wx[1, band], 0.0)                # nothing taken from the emptied layer
    psi0 = rng.uniform(0.0, 1.0, (3, g.N))
    out.update(a_h0=h0, a_u0=u0, a_theta0=theta0, a_nu4=nu4, a_nfast=nfast, a_wx=wx, a_psi0=psi0,
               a_cp=core.cpa, a_kappa=core.kap, a_rd=core.rda, a_drag=rcases.SURFACE_DRAG)
    M = h * cp.asarray(g.areaCell)[None]
    psi = cp.asarray(psi0)
    core.exchange(cp.asarray(wx), h, u, M, psi, theta=theta)
    out.update(a_h=h.get(), a_u=u.get(), a_M=M.get(), a_psi=psi.get(), a_theta=theta.get())
    return out


def air_theta(cp, g, dg, Layers, rcases, mycases):
    """The reference's air layers (Layers(air=...), step(..., theta=...)) from its aquaplanet start (cases.aqua: three
    layers at rest, theta 415 / 342.5 / 290 - 30 sin^2 phi K) over flat ground, the aqua preset's surface drag and
    nabla^4 (visc4_U 15), floor 10 kg/m^2, interfacial stress 5e-3 kg/m^2/s (so its heating, vmix_heat, runs too),
    dt 1800 s (the preset's at n = 4), nfast from the world's rule ceil(1.2 substeps) after update_gfast."""
    h0, b, u0, x = rcases.aqua(g)
    theta0 = x['theta']
    nu4 = mycases.visc4(g, 15.0)
    stress = [0.0, 0.0, rcases.SURFACE_DRAG]
    air = dict(t_ref=288.0)
    core = Layers(dg, 3, b=b, gprime=[0.0, 0.0], stress=stress, nu4=nu4, floor=10.0, air=air, vmix=5e-3)
    h, u, theta = cp.asarray(h0), cp.asarray(u0), cp.asarray(theta0)
    dt = 1800.0
    core.update_gfast(h, theta)
    gc0 = core.Gc.get()
    sub = core.substeps(h, dt)
    nfast = int(math.ceil(1.2 * sub))
    Fm = cp.zeros((3, g.E))
    d = dict(dt=dt, nfast=nfast, substeps=sub, nu4=nu4, stress=np.array(stress), floor=10.0, vmix=5e-3, h0=h0, u0=u0,
             theta0=theta0, b=b, Gc0=gc0, cp=core.cpa, kappa=core.kap, rd=core.rda)
    for st in range(1, 13):
        core.step(h, u, dt, nfast, Fm, theta=theta)
        if st == 1:
            d.update(h1=h.get(), u1=u.get(), theta1=theta.get(), Fm1=Fm.get())
    core.update_gfast(h, theta)
    d.update(h=h.get(), u=u.get(), theta=theta.get(), Fm=Fm.get(), Gc=core.Gc.get())
    return d


def vmix_heat(cp, g, dg, Layers, rcases):
    """The world's own call of the heating kernel from the layers' kernel table (world.py:317-318): after the sea
    coupling, the kinetic energy the wind stress removed over the tick (the sea's per-edge dissipation, J/m^2) returns
    as heat to the air layers' theta. Aquaplanet air layers (cases.aqua), seeded dissipation of the size a tick's wind
    stress gives (log-uniform 0.1 .. 1e4 J/m^2, zero on a tenth of the edges), two calls in a row."""
    from insilica.constants import P0
    from insilica.gpu import grid_dims
    h0, b, u0, x = rcases.aqua(g)
    core = Layers(dg, 3, b=b, gprime=[0.0, 0.0], floor=10.0, air=dict(t_ref=288.0), vmix=5e-3)
    rng = np.random.default_rng(11)
    diss = np.exp(rng.uniform(np.log(0.1), np.log(1e4), g.E)) * (rng.uniform(size=g.E) > 0.1)
    h, theta, dd = cp.asarray(h0), cp.asarray(x['theta']), cp.asarray(diss)
    grav = 9.80616
    d = dict(h=h0, diss=diss, theta0=x['theta'], grav=grav, cp=core.cpa, kappa=core.kap, p0=P0)
    i32, R = np.int32, np.float64
    for call in (1, 2):
        core.k['vmix_heat'](*grid_dims(g.N), (i32(g.N), i32(3), h, dd, dg.cellEdge, dg.le, dg.de, dg.areaCell, R(grav),
                                               R(core.cpa), R(core.kap), R(P0), theta))
        d[f'theta{call}'] = theta.get()
    return d


if __name__ == '__main__':
    main()
