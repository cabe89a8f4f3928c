"""Ensembles of stacked-layer members on one GPU (the reference's Ensemble, src/insilica/ensemble.py:8-29): every member
keeps its own state and does exactly what it does alone, and a step advances every member by one of its own steps.
Where the reference queues each member's captured tick graph on its own stream, here all members are stacks of one
isw.batch.Batch, so a step is one CUDA graph for the whole ensemble, whatever mix of grid levels it holds. Members of
different levels step with their own dt, so one ensemble step advances sum_i dt_i of model time."""
import numpy as np
import torch

from . import gpu
from . import grid as G
from .batch import Batch
from .workload import Member, planet_grid

SECONDS_PER_DAY = 86400.0


def device_grids(levels, device=0):
    """One DeviceGrid per distinct level (planet rotation as the stacked workloads use), in the current precision form."""
    out = {}
    for n in sorted(set(levels)):
        out[n] = gpu.DeviceGrid(planet_grid(G.build(n, device=device)), device=device)
    return out


class Ensemble:
    def __init__(self, members, batch):
        self.members = list(members)
        self.batch = batch

    @classmethod
    def build(cls, levels, seed=0, perturb=0.005, ntracers=2, precision='mixed', device=0, grids=None, kinds=('air', 'ocean')):
        """One member per entry of levels (member i seeded seed + i), all in one batch. grids: {level: DeviceGrid} to
        share grids across ensembles (built here otherwise, in the given precision form)."""
        prev = gpu.PRECISION
        gpu.set_precision(precision)
        try:
            grids = grids or device_grids(levels, device)
            batch = Batch(device)
            members = [Member(grids[n], seed + i, ntracers=ntracers, perturb=perturb, batch=batch, kinds=kinds,
                              init_device=torch.device(f'cuda:{device}'))
                       for i, n in enumerate(levels)]
        finally:
            gpu.set_precision(prev)
        return cls(members, batch)

    def step(self, k=1, stream=None):
        for _ in range(k):
            self.batch.step(stream)
        return self

    def member_days_per_step(self):
        return sum(m.dt for m in self.members) / SECONDS_PER_DAY

    def footprint(self):
        return sum(m.footprint() for m in self.members)

    def __iter__(self):
        return iter(self.members)

    def __len__(self):
        return len(self.members)
