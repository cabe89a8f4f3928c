"""The stacked-layer workloads as runnable objects: a Stack (one Layers + its Transport + device state) and the
two-stack member (an air stack of 3 layers and an ocean stack of 2, each with FCT tracers) that one model step of
the benchmark advances. State lives on the device; a step is one RK3 step of every stack, the receiving masses and
one FCT transport step of every tracer (reference world.py:290-301 for one stack)."""
import numpy as np
import torch

from . import cases
from .gpu import DeviceGrid
from .layers import Layers
from .transport import Transport

NFAST = 20


class Stack:
    def __init__(self, dg, state, dt, nfast=NFAST, ntracers=None, device=None):
        self.dg, self.dt, self.nfast = dg, float(dt), int(nfast)
        dev = torch.device(f'cuda:{dg.device}' if device is None else device)
        s = state
        self.L = s['L']
        self.core = Layers(dg, self.L, b=s['b'], gprime=s['gprime'], stress=s['stress'], nu4=s['nu4'], floor=s['floor'],
                           vmix=s.get('vmix', 0.0))
        tr = s['tracers'] if ntracers is None else s['tracers'][:ntracers]
        self.T = len(tr)
        self.tr = Transport(dg, layers=self.L, tracers=max(1, self.T))
        A = torch.as_tensor(dg.host.areaCell, dtype=torch.float64, device=dev)
        self.h = torch.as_tensor(np.ascontiguousarray(s['h']), dtype=torch.float64, device=dev)
        self.u = torch.as_tensor(np.ascontiguousarray(s['u']), dtype=torch.float64, device=dev)
        self.M = (self.h * A[None]).contiguous()
        self.M1 = torch.zeros_like(self.M)
        self.Fm = torch.zeros_like(self.u)
        self.tracers = [torch.as_tensor(np.ascontiguousarray(t), dtype=torch.float64, device=dev) for t in tr]

    def step(self, stream=None):
        self.core.step(self.h, self.u, self.dt, self.nfast, self.Fm, stream=stream)
        self.tr.mass_after(self.M, self.Fm, self.M1, stream=stream)
        if self.T:
            self.tr.step_many(self.M, self.M1, self.Fm, self.tracers, order=3, stream=stream)
        self.M, self.M1 = self.M1, self.M

    def state(self):
        return [self.h, self.u, self.M] + self.tracers

    def register(self, batch):
        """Add this stack to a Batch: the batch's step then does this stack's step(), with M <- M1 copied (not swapped)."""
        return batch.add(self.core, self.h, self.u, self.Fm, tr=self.tr if self.T else None, M=self.M, M1=self.M1,
                         tracers=self.tracers, dt=self.dt, nfast=self.nfast)

    def launches(self):
        """Kernels one step launches (csrc/layers.cu, csrc/transport.cu)."""
        n = sum(max(1, int(np.ceil(c * self.nfast))) for c in (1 / 3, 1 / 2, 1.0))
        k = 1 + (4 if self.core.nu4 else 0) + 3 * 5 + 2 * n + (1 if (self.core.vmix and self.L > 1) else 0)
        return k + 1 + (4 if self.T else 0)


class Member:
    """One benchmark member: the air and ocean stacks of one seed on one grid. batch: an isw.batch.Batch to register the
    stacks with (they are then advanced by Batch.step, all stacks in one launch); None steps them call by call."""

    def __init__(self, dg, seed, ntracers=3, perturb=0.01, dt=None, nfast=NFAST, batch=None):
        g = dg.host
        dt = cases.stack_dt(g.n) if dt is None else dt
        topo = cases.topography(g, seed)
        self.stacks = [Stack(dg, cases.stack_state(g, kind, seed, perturb=perturb, ntracers=ntracers, topo=topo), dt, nfast)
                       for kind in ('air', 'ocean')]
        self.dt = float(dt)
        self.batch, self.slots = batch, []
        if batch is not None:
            for s in self.stacks:
                self.slots.append(s.register(batch))

    def step(self, stream=None):
        if self.batch is not None:
            self.batch.step(stream)
            return
        for s in self.stacks:
            s.step(stream)

    def state(self):
        return [a for s in self.stacks for a in s.state()]

    def launches(self):
        """Kernels one step launches (in the batched case, the step graph's kernels, shared with the batch's other
        members)."""
        if self.batch is None:
            return sum(s.launches() for s in self.stacks)
        info = self.batch.info()
        n = sum(max(1, int(np.ceil(c * self.stacks[0].nfast))) for c in (1 / 3, 1 / 2, 1.0))
        nu4 = any(s.core.nu4 for s in self.stacks)
        return 1 + (3 if nu4 else 0) + 3 * 5 + (3 if info['tiles'] else 2 * n) + 4


def planet_grid(g, omega=cases.OMEGA_EARTH):
    """The grid with the stacked workloads' rotation (fV scaled, as the reference's for_planet does)."""
    from .grid import for_planet
    return for_planet(g, 6.371e6, omega, 9.80616)
