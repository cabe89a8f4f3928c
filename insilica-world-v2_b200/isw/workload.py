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

# Stacks that the mixed form runs in FP64, by grid level. Measured against the FP64 form over 10 model days
# (isw.accuracy.member): every stack of the mixed form stays within 1e-5 relative L2 in h and u except the ocean stack at
# levels 4 and 5, whose jet over the coarse grid amplifies any perturbation by ~2.6x per model day: the FP64 form itself,
# started from h x (1 + 1e-8 r), ends 1e-6 (h) and 1e-5 .. 1e-4 (u) away after 10 days, so FP32 momentum's rounding
# (1e-7 relative per step in the balanced PV flux and pressure gradient) ends at 1e-5 .. 6e-4. Those stacks run in the
# FP64 form inside mixed batches (a batch holds stacks of both forms); the air stacks and every finer level stay mixed.
FP64_IN_MIXED = {4: ('ocean',), 5: ('ocean',)}


def fp64_stack_kinds(level):
    """The stack kinds a mixed-form member at this grid level runs in the FP64 form."""
    return FP64_IN_MIXED.get(int(level), ())


class Stack:
    def __init__(self, dg, state, dt, nfast=NFAST, ntracers=None, device=None, precision=None):
        """precision: 'double' or 'mixed' for this stack's Layers and Transport; None takes the grid's form."""
        self.dg, self.dt, self.nfast = dg, float(dt), int(nfast)
        dev = torch.device(f'cuda:{dg.device}' if device is None else device)
        s = state
        self.L = s['L']
        self.kind = s.get('kind')
        self.core = Layers(dg, self.L, b=s['b'], gprime=s['gprime'], stress=s['stress'], nu4=s['nu4'], floor=s['floor'],
                           vmix=s.get('vmix', 0.0), vmix_cd=s.get('vmix_cd', 0.0), precision=precision)
        tr = s['tracers'] if ntracers is None else s['tracers'][:ntracers]
        self.T = len(tr)
        self.tr = Transport(dg, layers=self.L, tracers=max(1, self.T), precision=precision)
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

    def arrays(self, prefix):
        """The stack's resident state as host arrays named prefix + h, u, M, tr0.. (for a save file)."""
        out = {prefix + 'h': self.h.cpu().numpy(), prefix + 'u': self.u.cpu().numpy(), prefix + 'M': self.M.cpu().numpy()}
        out.update({f'{prefix}tr{j}': t.cpu().numpy() for j, t in enumerate(self.tracers)})
        return out

    def load(self, arrays, prefix):
        """Overwrite the resident state from arrays (as written by arrays())."""
        for name, t in [('h', self.h), ('u', self.u), ('M', self.M)] + [(f'tr{j}', x) for j, x in enumerate(self.tracers)]:
            t.copy_(torch.as_tensor(arrays[prefix + name], device=t.device))

    def reset(self, state):
        """Start this stack over from a new initial state of the same kind (a stack_state dict for the same grid, layer
        count and tracers): h, u, the tracers and the bottom from the state, M = h x area, M1 and Fm cleared. The Layers
        and Transport objects and every device array are kept."""
        s = state
        dev = self.h.device
        self.h.copy_(torch.as_tensor(np.ascontiguousarray(s['h']), dtype=torch.float64, device=dev))
        self.u.copy_(torch.as_tensor(np.ascontiguousarray(s['u']), dtype=torch.float64, device=dev))
        A = torch.as_tensor(self.dg.host.areaCell, dtype=torch.float64, device=dev)
        self.M.copy_(self.h * A[None])
        self.M1.zero_()
        self.Fm.zero_()
        for t, x in zip(self.tracers, s['tracers']):
            t.copy_(torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=dev))
        self.core.set_bottom(s['b'])

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
    """One benchmark member: the air and ocean stacks of one seed on one grid (kinds=('air',) for the 3-layer form).
    batch: an isw.batch.Batch to register the stacks with (they are then advanced by Batch.step, all stacks in one
    launch); None steps them call by call. init_device: synthesise the random initial fields on that CUDA device.
    fp64_kinds: the stack kinds to run in the FP64 form when the grid's form is mixed; None applies FP64_IN_MIXED, ()
    keeps every stack mixed."""

    def __init__(self, dg, seed, ntracers=3, perturb=0.01, dt=None, nfast=NFAST, batch=None, kinds=('air', 'ocean'),
                 init_device=None, fp64_kinds=None):
        g = dg.host
        dt = cases.stack_dt(g.n) if dt is None else dt
        topo = cases.topography(g, seed, device=init_device)
        fk = _fp64_kinds(dg, fp64_kinds)
        self.stacks = [Stack(dg, cases.stack_state(g, kind, seed, perturb=perturb, ntracers=ntracers, topo=topo,
                                                   device=init_device), dt, nfast,
                             precision='double' if kind in fk else None)
                       for kind in kinds]
        self.dt = float(dt)
        self.batch, self.slots = batch, []
        if batch is not None:
            for s in self.stacks:
                self.slots.append(s.register(batch))

    @classmethod
    def from_states(cls, dg, states, dt=None, nfast=NFAST, batch=None, fp64_kinds=None):
        """A member from prepared stack states (cases.stack_state dicts), e.g. initial conditions that came with a
        request; nothing is synthesised here. fp64_kinds as for the constructor."""
        self = cls.__new__(cls)
        dt = cases.stack_dt(dg.host.n) if dt is None else dt
        fk = _fp64_kinds(dg, fp64_kinds)
        self.stacks = [Stack(dg, s, dt, nfast, precision='double' if s.get('kind') in fk else None) for s in states]
        self.dt = float(dt)
        self.batch, self.slots = batch, []
        if batch is not None:
            for s in self.stacks:
                self.slots.append(s.register(batch))
        return self

    def step(self, stream=None):
        if self.batch is not None:
            self.batch.step(stream)
            return
        for s in self.stacks:
            s.step(stream)

    def state(self):
        return [a for s in self.stacks for a in s.state()]

    def finite(self):
        """Whether every stack's thicknesses are finite (a device reduction; synchronises)."""
        return all(bool(torch.isfinite(s.h).all()) for s in self.stacks)

    def reset(self, states, batch=None):
        """Reuse this member for new initial states of the same kinds (Stack.reset), registered with `batch` if given."""
        for st, s in zip(self.stacks, states):
            st.reset(s)
        if batch is not None:
            self.batch, self.slots = batch, [st.register(batch) for st in self.stacks]

    def unregister(self):
        if self.batch is not None:
            for slot in self.slots:
                self.batch.remove(slot)
        self.batch, self.slots = None, []

    def footprint(self):
        """Device bytes this member holds: its state arrays and the scratch of its Layers and Transport objects."""
        return sum(stack_bytes(s.dg.host, s.L, s.T, s.core.precision == 1) for s in self.stacks)

    def launches(self):
        """Kernels one step launches (in the batched case, the step graph's kernels, shared with the batch's other
        members)."""
        if self.batch is None:
            return sum(s.launches() for s in self.stacks)
        info = self.batch.info()
        n = sum(max(1, int(np.ceil(c * self.stacks[0].nfast))) for c in (1 / 3, 1 / 2, 1.0))
        nu4 = any(s.core.nu4 for s in self.stacks)
        tr = any(s.T for s in self.stacks)
        fast = 3 * info['groups'] if info['tiles'] else (3 if info['persistent'] else 2 * n)
        return 1 + (3 if nu4 else 0) + 3 * 5 + fast + 1 + (6 if tr else 0)


def _fp64_kinds(dg, fp64_kinds):
    if not dg.mixed:
        return ()
    return fp64_stack_kinds(dg.host.n) if fp64_kinds is None else tuple(fp64_kinds)


def planet_grid(g, omega=cases.OMEGA_EARTH):
    """The grid with the stacked workloads' rotation (fV scaled, as the reference's for_planet does)."""
    from .grid import for_planet
    return for_planet(g, 6.371e6, omega, 9.80616)


def stack_bytes(g, L, T, mixed):
    """Device bytes of one stack on grid g: state (h, u, Fm, M, M1, T tracers), the Layers scratch (csrc/layers.cu
    layers_create; the mixed form's FP32 scratch too) and the Transport scratch (csrc/transport.cu)."""
    N, E, NV = g.N, g.E, g.NV
    R = max(1, T) * L
    doubles = 3 * L * N + 2 * L * E + T * L * N
    doubles += 11 * N + NV + 5 * L * N + 2 * L * NV + 10 * L * E + 8 * E
    doubles += 6 * R * N + R * E
    floats = 0
    if mixed:
        floats += 11 * L * E + 2 * L * N + 2 * L * NV + 6 * E + 12 * N
        floats += 4 * R * N + R * E
    return 8 * doubles + 4 * floats
