"""Accuracy of the mixed precision form against the plain FP64 form (which the parity tests hold to the reference):
the error norms of the reference's accuracy test (reference tests/test_accuracy.py:21-23 l2rel, :45-49 vertex
vorticity) and mass drifts by the deterministic sum.

- member(level, days): the stacked benchmark member (air 3 + ocean 2 layers, 3 tracers) in both forms from the same
  state; per stack the relative L2 (area-weighted) and Linf errors of h and u after `days`, and the relative drift of
  every layer's volume and every tracer's mass over the run, in both forms. The mixed member runs its stacks as
  mixed-form ensembles and serving do (the ocean stack at levels 4 and 5 in FP64: workload.FP64_IN_MIXED);
  fp64_kinds=() measures the mixed form on every stack.
- galewsky(level, days): the Galewsky jet (one layer, the reference's initial state) in both forms; L2/Linf of vertex
  vorticity and of h, and the mass drift.
- w2(level, days): Williamson 2 (one layer, steady solid-body flow, dt 900 s at level 4) in both forms: h and u
  errors and the mass drift."""
import numpy as np
import torch

from . import cases, gpu
from . import grid as G
from .batch import Batch
from .layers import Layers
from .workload import Member, planet_grid

SECONDS_PER_DAY = 86400.0


def l2rel(area, a, b):
    return float(np.sqrt(np.sum(area * (a - b) ** 2) / np.sum(area * b ** 2)))


def linf(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def vertex_vorticity(g, u):
    z = np.zeros(g.NV)
    np.add.at(z, g.ev1, g.circ1 * g.de * u)
    np.add.at(z, g.ev2, g.circ2 * g.de * u)
    return z / g.areaV


def _masses(stack):
    A = torch.as_tensor(stack.dg.host.areaCell, device=stack.h.device)
    vol = [gpu.dsum(stack.h[k], A) for k in range(stack.L)]
    trm = [gpu.dsum(t[k], stack.M[k]) for t in stack.tracers for k in range(stack.L)]
    return np.array(vol), np.array(trm)


def member(level=6, days=10.0, seed=0, device=0, fp64_kinds=None, tiles=None):
    g = planet_grid(G.build(level, device=device))
    forms = {}
    for prec in ('double', 'mixed'):
        gpu.set_precision(prec)
        try:
            dg = gpu.DeviceGrid(g, device=device)
        finally:
            gpu.set_precision('double')
        b = Batch(device)
        if tiles is not None:                  # the fast loop in tiles or in grid-wide passes (None: the default)
            b.config(tiles=tiles)
        m = Member(dg, seed, batch=b, fp64_kinds=fp64_kinds)
        forms[prec] = (m, b, [_masses(s) for s in m.stacks])
    steps = int(round(days * SECONDS_PER_DAY / forms['double'][0].dt))
    for _ in range(steps):
        for m, b, _ in forms.values():
            b.step()
    torch.cuda.synchronize()
    out = dict(level=level, days=days, steps=steps, stacks=[])
    for k, name in enumerate(('air', 'ocean')):
        sd, sm = forms['double'][0].stacks[k], forms['mixed'][0].stacks[k]
        area = g.areaCell
        hd, hm, ud, um = sd.h.cpu().numpy(), sm.h.cpu().numpy(), sd.u.cpu().numpy(), sm.u.cpu().numpy()
        le_de = g.le * g.de                        # the edge area weight l_e d_e / 2 (the constant 1/2 cancels)
        row = dict(stack=name, L=sd.L, form='double' if sm.core.precision == 0 else 'mixed',
                   h_l2=l2rel(area[None], hm, hd), h_linf=linf(hm, hd),
                   u_l2=l2rel(le_de[None], um, ud), u_linf=linf(um, ud),
                   h_rel_l2_plain=float(np.linalg.norm(hm - hd) / np.linalg.norm(hd)),
                   u_rel_l2_plain=float(np.linalg.norm(um - ud) / np.linalg.norm(ud)))
        for prec in ('double', 'mixed'):
            s = forms[prec][0].stacks[k]
            v0, t0 = forms[prec][2][k]
            v1, t1 = _masses(s)
            row[f'volume_drift_{prec}'] = float(np.max(np.abs(v1 - v0) / np.abs(v0)))
            row[f'tracer_mass_drift_{prec}'] = float(np.max(np.abs(t1 - t0) / np.abs(t0)))
        out['stacks'].append(row)
    out['status'] = [b.status() for _, b, _ in forms.values()]
    return out


def galewsky(level=7, days=6.0, nfast=2, device=0):
    g = G.for_planet(G.build(level, device=device), 6.371e6, 7.292e-5, 9.80616)
    h0, bt, u0 = cases.initial_state(g, 'galewsky')
    dt = cases.default_dt(level)
    A = torch.as_tensor(g.areaCell, device=f'cuda:{device}')
    res = {}
    for prec in ('double', 'mixed'):
        gpu.set_precision(prec)
        try:
            core = Layers(gpu.DeviceGrid(g, device=device), 1, b=bt)
        finally:
            gpu.set_precision('double')
        h = torch.as_tensor(np.ascontiguousarray(h0[None]), device=f'cuda:{device}')
        u = torch.as_tensor(np.ascontiguousarray(u0[None]), device=f'cuda:{device}')
        b = Batch(device)
        b.add(core, h, u, torch.zeros_like(u), dt=dt, nfast=nfast)
        m0 = gpu.dsum(h[0], A)
        steps = int(round(days * SECONDS_PER_DAY / dt))
        for _ in range(steps):
            b.step()
        torch.cuda.synchronize()
        res[prec] = (h.cpu().numpy()[0], u.cpu().numpy()[0], (gpu.dsum(h[0], A) - m0) / m0, b.status(), steps)
    hd, ud, dd, _, steps = res['double']
    hm, um, dm, _, _ = res['mixed']
    zd, zm = vertex_vorticity(g, ud), vertex_vorticity(g, um)
    return dict(level=level, days=days, steps=steps, dt=dt, nfast=nfast,
                vorticity_l2=l2rel(g.areaV, zm, zd), vorticity_linf=linf(zm, zd),
                h_l2=l2rel(g.areaCell, hm, hd), h_linf=linf(hm, hd),
                mass_drift_mixed=float(dm), mass_drift_double=float(dd),
                status=[res['double'][3], res['mixed'][3]])


def w2(level=4, days=5.0, device=0):
    g = G.for_planet(G.build(level, device=device), 6.371e6, 7.292e-5, 9.80616)
    h0, bt, u0 = cases.initial_state(g, 'w2')
    dt, nfast = 900.0 * 2.0 ** (4 - level), 2
    A = torch.as_tensor(g.areaCell, device=f'cuda:{device}')
    res = {}
    for prec in ('double', 'mixed'):
        gpu.set_precision(prec)
        try:
            core = Layers(gpu.DeviceGrid(g, device=device), 1, b=bt)
        finally:
            gpu.set_precision('double')
        h = torch.as_tensor(np.ascontiguousarray(h0[None]), device=f'cuda:{device}')
        u = torch.as_tensor(np.ascontiguousarray(u0[None]), device=f'cuda:{device}')
        b = Batch(device)
        b.add(core, h, u, torch.zeros_like(u), dt=dt, nfast=nfast)
        m0 = gpu.dsum(h[0], A)
        steps = int(round(days * SECONDS_PER_DAY / dt))
        for _ in range(steps):
            b.step()
        torch.cuda.synchronize()
        res[prec] = (h.cpu().numpy()[0], u.cpu().numpy()[0], (gpu.dsum(h[0], A) - m0) / m0, steps)
    hd, ud, dd, steps = res['double']
    hm, um, dm, _ = res['mixed']
    le_de = g.le * g.de
    return dict(level=level, days=days, steps=steps, h_l2=l2rel(g.areaCell, hm, hd), u_l2=l2rel(le_de, um, ud),
                h_linf=linf(hm, hd), u_linf=linf(um, ud), mass_drift_mixed=float(dm), mass_drift_double=float(dd))
