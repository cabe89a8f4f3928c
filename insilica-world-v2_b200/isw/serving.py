"""A forecast server on one GPU with continuous batching: requests (a grid level, a horizon in model days, 3 or 5 layers)
arrive over time; each is admitted as soon as its device footprint fits the memory budget (and a slot is free), its
state is created on the device and registered with the server's batch, and from then on every batched step advances it
together with every other admitted request, each by one of its own steps. A request that reaches its horizon is copied
back to the host and released at once, and the requests waiting for memory are admitted in arrival order. State stays
resident on the device from admission to completion; nothing is copied between steps.

A request's result does not depend on what else is in the batch: every stack's arithmetic is its own (the batched
kernels give each stack the same operations in the same order whatever shares the launch).

The request stream of the benchmark: seeded Poisson arrivals at `rate` requests per second of the server's wall clock,
the level uniform over 4..7, the horizon log-uniform over 1..30 model days, 3 (air) or 5 (air and ocean) layers, initial
states as the stacked benchmark member's (seed = request id), carried by the requests (Server.prepare) as a client's
analysis would be; admission allocates the request's device state and uploads it."""
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, gpu
from .batch import Batch
from .ensemble import device_grids
from .workload import Member, fp64_stack_kinds, stack_bytes

SECONDS_PER_DAY = 86400.0


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the run
    level: int
    days: float
    layers: int             # 3: the air stack; 5: air and ocean
    seed: int = 0
    state: list = field(default=None, repr=False)   # the initial stack states (host), as a client sends them
    resume: dict = field(default=None, repr=False)  # a checkpoint to continue from: arrays and steps left


@dataclass
class Result:
    rid: int
    level: int
    layers: int
    days: float
    steps: int
    arrival: float
    admitted: float
    done: float
    state: list = field(default_factory=list, repr=False)   # host copies of h, u (and M, tracers) per stack
    error: str = ''         # empty for a completed forecast; else why the request was dropped

    @property
    def latency(self):
        return self.done - self.arrival


def poisson_requests(n, rate, seed=0, levels=(4, 5, 6, 7), days=(1.0, 30.0), layers=(3, 5)):
    """n requests: exponential gaps of mean 1/rate seconds, level uniform over `levels`, horizon log-uniform over `days`,
    layers uniform over `layers` (seeded)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    lv = rng.choice(levels, n)
    hz = np.exp(rng.uniform(math.log(days[0]), math.log(days[1]), n))
    ly = rng.choice(layers, n)
    return [Request(i, float(t[i]), int(lv[i]), float(hz[i]), int(ly[i]), seed=1000 + i) for i in range(n)]


def request_bytes(g, layers, ntracers, mixed):
    """Device bytes of a request's member; in the mixed form the stacks FP64_IN_MIXED names for the level are FP64."""
    kinds = ('air',) if layers == 3 else ('air', 'ocean')
    fk = fp64_stack_kinds(g.n) if mixed else ()
    return sum(stack_bytes(g, 3 if k == 'air' else 2, ntracers, mixed and k not in fk) for k in kinds)


class Server:
    def __init__(self, device=0, budget_bytes=150e9, precision='mixed', ntracers=2, max_active=256, grids=None,
                 keep_state=False):
        self.device = int(device)
        self.dev = torch.device(f'cuda:{self.device}')
        self.budget = float(budget_bytes)
        self.precision = precision
        self.ntracers = ntracers
        self.max_active = max_active
        self.keep_state = keep_state
        self.grids = grids or {}
        self.batch = Batch(self.device)
        # members of finished requests, kept resident per (level, layers) and reused for the next request of that kind
        # (its state, terrain and tracers loaded into them): admission then allocates nothing, completion frees nothing
        self._pool = {}
        # a serving batch changes at every admission and completion, and most of its steps run few requests: grid-wide
        # sub-steps need no tiles rebuilt for each new mix, and two launches per sub-step beat the persistent loop for
        # small batches (8 level-6 members: 2.82 against 3.22 ms a step)
        self.batch.config(tiles=False, persistent=False)

    def _grid(self, level):
        if level not in self.grids:
            prev = gpu.PRECISION
            gpu.set_precision(self.precision)
            try:
                self.grids.update(device_grids([level], self.device))
            finally:
                gpu.set_precision(prev)
        return self.grids[level]

    def prepare(self, requests):
        """Give every request its initial state (the stacked benchmark member's, seeded by the request), synthesised on
        the device: what a client would send with the request. Done before a timed run."""
        from . import cases
        for r in requests:
            if r.state is None:
                g = self._grid(r.level).host
                topo = cases.topography(g, r.seed, device=self.dev)
                kinds = ('air',) if r.layers == 3 else ('air', 'ocean')
                r.state = [cases.stack_state(g, k, r.seed, perturb=0.01, ntracers=self.ntracers, topo=topo, device=self.dev)
                           for k in kinds]

    def footprint(self, req):
        return request_bytes(self._grid(req.level).host, req.layers, self.ntracers, self.precision == 'mixed')

    def _admit(self, req, now):
        prev = gpu.PRECISION
        gpu.set_precision(self.precision)
        try:
            if req.state is None:
                self.prepare([req])
            pool = self._pool.get((req.level, req.layers))
            if pool:
                m = pool.pop()
                m.reset(req.state, batch=self.batch)
            else:
                m = Member.from_states(self._grid(req.level), req.state, batch=self.batch)
        finally:
            gpu.set_precision(prev)
        steps = max(1, int(math.ceil(req.days * SECONDS_PER_DAY / m.dt - 1e-9)))
        left = steps
        if req.resume is not None:                  # continue a checkpointed run from its saved state
            for k, st in enumerate(m.stacks):
                st.load(req.resume['arrays'], f's{k}_')
            left = int(req.resume['left'])
        return dict(req=req, member=m, left=left, steps=steps, admitted=now, bytes=self.footprint(req))

    def checkpoint(self, directory, active, waiting):
        """Write every resident request's state (reference save-file format: isw.savefile) and the waiting requests'
        descriptions to `directory`; Server.resume reads them back."""
        import json
        from pathlib import Path
        from . import savefile
        d = Path(directory)
        d.mkdir(parents=True, exist_ok=True)
        files = []
        for a in active:
            r, m = a['req'], a['member']
            arrays = {}
            for k, st in enumerate(m.stacks):
                arrays.update(st.arrays(f's{k}_'))
            meta = dict(rid=r.rid, arrival=r.arrival, level=r.level, days=r.days, layers=r.layers, seed=r.seed,
                        steps=a['steps'], left=a['left'], precision=self.precision, ntracers=self.ntracers)
            name = f'request_{r.rid}.zip'
            savefile.write(d / name, meta, arrays)
            files.append(name)
        pending = [dict(rid=r.rid, arrival=r.arrival, level=r.level, days=r.days, layers=r.layers, seed=r.seed) for r in waiting]
        (d / 'manifest.json').write_text(json.dumps(dict(resident=files, waiting=pending), indent=1, sort_keys=True))

    @staticmethod
    def resume(directory):
        """The requests of a checkpoint (Server.checkpoint): resident ones carry their saved state and steps left,
        waiting ones start from their seeds; all arrive at time 0 of the next run."""
        import json
        from pathlib import Path
        from . import savefile
        d = Path(directory)
        man = json.loads((d / 'manifest.json').read_text())
        out = []
        for name in man['resident']:
            meta, arrays = savefile.read(d / name)
            out.append(Request(meta['rid'], 0.0, meta['level'], meta['days'], meta['layers'], seed=meta['seed'],
                               resume=dict(arrays=arrays, left=meta['left'])))
        for w in man['waiting']:
            out.append(Request(w['rid'], 0.0, w['level'], w['days'], w['layers'], seed=w['seed']))
        return out

    def run(self, requests, stream=None, clock=time.perf_counter, stop_after=None, checkpoint_dir=None):
        """Serve the requests (arrival times relative to the start of the call); returns (results in completion order,
        stats). A request is done when its final state is on the host. stop_after: after that many batched steps,
        checkpoint the resident and waiting requests to checkpoint_dir and return (Server.resume continues them)."""
        st = torch.cuda.current_stream(self.dev) if stream is None else stream
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting, active, results = deque(), [], []
        used = 0.0
        pooled = sum(len(v) * self.footprint(Request(0, 0.0, k[0], 0.0, k[1])) for k, v in self._pool.items())
        steps = 0
        model_days = 0.0
        admit_s = step_s = 0.0                              # wall time admitting requests and running batched steps
        t0 = clock()
        while pending or waiting or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            while waiting and len(active) < self.max_active:
                req = waiting[0]
                need = self.footprint(req)
                reuse = bool(self._pool.get((req.level, req.layers)))
                if not reuse:                               # free pooled members of other kinds while memory is short
                    while used + pooled + need > self.budget and any(self._pool.values()):
                        key = next(k for k, v in self._pool.items() if v)
                        self._pool[key].pop()
                        pooled -= self.footprint(Request(0, 0.0, key[0], 0.0, key[1]))
                if used + (0 if reuse else pooled) + need > self.budget and active:
                    break                                   # wait for memory (a lone request is always admitted)
                if reuse:
                    pooled -= need
                waiting.popleft()
                ta = clock()
                a = self._admit(req, ta - t0)
                admit_s += clock() - ta
                used += a['bytes']
                active.append(a)
            if not active:
                if pending:                                 # idle until the next arrival
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (clock() - t0))))
                continue
            if stop_after is not None and steps >= stop_after:
                self.checkpoint(checkpoint_dir, active, list(waiting) + list(pending))
                for a in active:
                    a['member'].unregister()
                active = []
                break
            ts = clock()
            self.batch.step(st)
            st.synchronize()
            step_s += clock() - ts
            steps += 1
            code = self.batch.status(stream=st)             # the host mirror of the status word: no device sync
            if code == _lib.ISW_ENOTFINITE:
                # a forecast whose state went non-finite: drop it with an error result; the step ran every other stack
                # to completion with its own arithmetic, so they carry on once the status is cleared
                for a in [a for a in active if not a['member'].finite()]:
                    a['member'].unregister()
                    active.remove(a)
                    used -= a['bytes']
                    req = a['req']
                    results.append(Result(req.rid, req.level, req.layers, req.days, a['steps'], req.arrival, a['admitted'],
                                          clock() - t0, error=f'non-finite thickness after {a["steps"] - a["left"] + 1} steps'))
                self.batch.status(reset=True, stream=st)
            elif code != 0:
                raise _lib.IswError(code, 'serving: the batched step reported a failure; results withheld')
            finished = []
            for a in active:
                a['left'] -= 1
                model_days += a['member'].dt / SECONDS_PER_DAY
                if a['left'] == 0:
                    finished.append(a)
            for a in finished:
                m, req = a['member'], a['req']
                m.unregister()
                state = [x.cpu() for x in m.state()] if self.keep_state else [x.cpu() for x in m.state()[:2]]
                active.remove(a)
                used -= a['bytes']
                self._pool.setdefault((req.level, req.layers), []).append(m)
                pooled += a['bytes']
                results.append(Result(req.rid, req.level, req.layers, req.days, a['steps'], req.arrival, a['admitted'],
                                      clock() - t0, state if self.keep_state else []))
                del m, a
        wall = clock() - t0
        done = [r for r in results if not r.error]
        lat = np.array([r.latency for r in done]) if done else np.zeros(1)
        stats = dict(requests=len(done), failed=len(results) - len(done), batched_steps=steps, wall_s=wall, admit_s=admit_s,
                     step_s=step_s, model_days=model_days,
                     member_days_per_s=model_days / wall if wall > 0 else 0.0,
                     p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)), max_s=float(lat.max()))
        return results, stats


def sequential_baseline(requests, step_seconds, days_of):
    """The same requests served one at a time in arrival order (FIFO, one server) by a core whose step takes
    step_seconds[(level, layers)] seconds: completion times by the single-server queue recursion, latencies, and the
    member-days per second of service time. days_of(req) gives (steps, model days)."""
    t, lat, busy, days = 0.0, [], 0.0, 0.0
    for r in sorted(requests, key=lambda r: r.arrival):
        n, d = days_of(r)
        service = n * step_seconds[(r.level, r.layers)]
        t = max(t, r.arrival) + service
        lat.append(t - r.arrival)
        busy += service
        days += d
    lat = np.array(lat)
    return dict(p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)), wall_s=t,
                member_days_per_s=days / busy if busy > 0 else 0.0)
