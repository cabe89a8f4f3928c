"""Benchmark: model days per second of the stacked-layer TRiSK step with FCT transport at level 6.

Workload (one "step"): the level-6 member of the stacked-layer benchmark, an air stack of 3 Boussinesq layers and an
ocean stack of 2 (40962 cells, 122880 edges, 81920 vertices), each advanced by one time-split RK3 step (nfast = 20,
37 barotropic sub-steps, hyperviscosity, interfacial stress), its receiving masses and one FCT transport step of 3
tracers. dt = 300 s, so a step is 300 s of model time. Synthetic seeded initial states (balanced jets, random
spherical-harmonic terrain, 1% perturbations, random tracers); the grid is built on the device (Lloyd to 1e-11 rad).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl isw|reference] [--level 6]
    python bench.py --workload ensemble    # 64 members (40 at level 5, 16 at 6, 8 at 7), mixed form: member-days/s
    python bench.py --workload serving     # Poisson request stream with continuous batching: p50/p99, member-days/s
    python bench.py --workload accuracy    # mixed form against FP64: level-6 member 10 days, level-7 Galewsky 6 days
    python bench.py --workload profile --form double|mixed --steps 5   # untimed steps, for ncu launch lists

On one GPU the line also carries `level7` (the same member at level 7, beyond the L2, both forms), `ensemble` (the
64-member mixed ensemble, a few timed steps, with the sequential FP64 loop beside it) and `serving` (a shortened
Poisson stream); `--no-configs` leaves them out.

Under torchrun (N > 1) every rank advances its own member (replicas: the members are independent) and rank 0 prints
one JSON line with the whole job's model days per second (the max step time over ranks); `--gpus N` without torchrun
starts the N ranks itself. `--impl reference` times the reference's own kernels compiled for the host (oracle/_ref),
driven through the reference's step sequence on the reference's own level-6 grid, on the host cores, rank 0 only.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / 'insilica-world-v2_b200'))

import numpy as np  # noqa: E402

L2_BYTES = 126 * 2 ** 20
SECONDS_PER_DAY = 86400.0


def peaks():
    p = ROOT / 'MEASURED_PEAKS.json'
    if p.exists():
        d = json.loads(p.read_text())
        return float(d['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


def metric_name(level):
    return f'model days/s, level {level}, air (3 layers) + ocean (2 layers) stacks, FCT 3 tracers each, nfast 20'


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.Q}', '--format=csv,noheader,nounits',
                                          '-lms', '200'], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(',')])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        if not self.rows:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled']}
        sm = [float(r[1]) for r in self.rows if r[1].replace('.', '', 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace('.', '', 1).isdigit()]
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.lower() == 'active'})
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': max(mx) if mx else None, 'reasons': reasons,
                'samples': len(self.rows)}


def build_grid(level, device):
    from isw import grid as G
    from isw.workload import planet_grid
    t = time.time()
    g = G.build(level, device=device)
    return planet_grid(g), time.time() - t


def cpu_member(g, seed, backend):
    """The same member on the host, through the oracle driver (backend 'oracle': this project's C restatement;
    'reference': the reference's own kernels compiled for the host)."""
    from isw import cases
    from oracle import model as M
    og = M.OracleGrid(g)
    stacks = []
    topo = cases.topography(g, seed)
    for kind in ('air', 'ocean'):
        s = cases.stack_state(g, kind, seed, ntracers=3, topo=topo)
        core = M.Layers(og, s['L'], b=s['b'], gprime=s['gprime'], stress=s['stress'], nu4=s['nu4'], floor=s['floor'],
                        vmix=s['vmix'], vmix_cd=s.get('vmix_cd', 0.0), backend=backend)
        tr = M.Transport(og, layers=s['L'], tracers=3, backend=backend)
        h, u = s['h'].copy(), s['u'].copy()
        Mm = h * g.areaCell[None]
        stacks.append(dict(core=core, tr=tr, h=h, u=u, M=Mm, M1=np.zeros_like(Mm), Fm=np.zeros_like(u),
                           trc=[t.copy() for t in s['tracers']]))
    dt = cases.stack_dt(g.n)

    def step():
        for s in stacks:
            s['core'].step(s['h'], s['u'], dt, 20, s['Fm'])
            s['tr'].mass_after(s['M'], s['Fm'], s['M1'])
            s['tr'].step_many(s['M'], s['M1'], s['Fm'], s['trc'], order=3)
            s['M'], s['M1'] = s['M1'], s['M']
    step.state = lambda: [a for s in stacks for a in [s['h'], s['u'], s['M']] + s['trc']]   # Member.state() order
    return step, dt


def time_cpu(step, budget_s, max_steps):
    """Mean seconds per step over a bounded sample (at least one step, at most max_steps or budget_s)."""
    step()                                   # warm the caches and the thread pool
    n, t0 = 0, time.perf_counter()
    while n < max_steps and (n == 0 or time.perf_counter() - t0 < budget_s):
        step()
        n += 1
    return (time.perf_counter() - t0) / n, n


def ensure_oracle():
    from oracle import model as M
    if not (ROOT / 'oracle' / 'liboracle.so').exists():
        M.build()


def member_config(args, g, world):
    """The `config` of the member workload: the same dict in both arms, so their lines describe one workload."""
    return dict(workload=f'level-{args.level} member: air 3 + ocean 2 layers, 3 tracers each, nfast 20, dt 300 s',
                level=args.level, cells=int(g.N), edges=int(g.E), vertices=int(g.NV), parallelism=f'replicas x{world}',
                l2='GPU arm: L2 flushed between timed steps (252 MB write); CPU arm: no GPU cache involved')


def reference_grid(level):
    """The reference's own level-n grid (oracle/_ref, built by its Python from its Lloyd positions), with the workload's
    rotation; None where it was not built. Host arrays only: nothing of isw's device code is loaded."""
    from oracle import build_ref
    p = build_ref.grid_path(level)
    if not p.exists():
        return None
    from isw import grid as G                # host-side container (NumPy), no device library
    return G.for_planet(G.load(p), 6.371e6, 7.292e-5, 9.80616)


def run_reference(args, rank, world):
    """The reference arm: its own kernels (oracle/_ref, built for the host) in its step sequence, on its own grid
    (oracle/_ref/grid_n<level>.npz), on the host cores, rank 0 only. Loads nothing of isw's device library."""
    if rank != 0:
        return
    from oracle import refkernels
    threads = os.cpu_count() or 1
    out = dict(metric=metric_name(args.level), unit='model days/s', impl='reference', n_gpus=world, steps=args.steps,
               warmup=args.warmup, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f64', data='synthetic')
    g = reference_grid(args.level) if refkernels.available() else None
    if g is None:
        out['unavailable'] = ('oracle/_ref was not built (the reference sources were absent when build() ran)'
                              if not refkernels.available() else f'oracle/_ref/grid_n{args.level}.npz was not built')
        print(json.dumps(out), flush=True)
        return
    out['config'] = member_config(args, g, world)
    ensure_oracle()
    step, dt = cpu_member(g, 0, 'reference')
    for _ in range(max(0, min(args.warmup, 1))):
        step()
    sec, n = time_cpu(step, budget_s=max(20.0, 2.0 * args.steps), max_steps=args.steps)
    v = dt / SECONDS_PER_DAY / sec
    out.update(value=v, ms_per_step=sec * 1e3,
               cpu_baseline=dict(value=v, unit='model days/s', cores=threads, kind='reference',
                                 sample=f'{n} full steps of the workload (reference kernels compiled for the host, OpenMP over '
                                        f'blocks, on the reference-built level-{args.level} grid)'),
               e2e=dict(value=v, unit='model days/s', h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(out), flush=True)


def member_status(m):
    """The failure status of the batch a member steps through (0 when none, or when it steps call by call)."""
    if m is None or getattr(m, 'batch', None) is None:
        return 0
    return m.batch.status()


def max_over_ranks(x, dist, device):
    """The largest of every rank's x (a time: the job runs at its slowest rank's pace); x itself without a process
    group. Every rank takes this collective at the same point."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, dt, ms):
    """Model days per second of the whole job: `world` replicas, each advancing dt seconds of model time per step of
    ms milliseconds (the max over ranks)."""
    return world * (dt / SECONDS_PER_DAY) / (ms / 1e3)


def free_port():
    import socket
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def spawn_ranks(n):
    """Run this benchmark as n ranks on one node (torch.distributed.run, rendezvous on 127.0.0.1); its exit code."""
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1', f'--nproc-per-node={n}', '--master-addr', '127.0.0.1',
           '--master-port', str(free_port()), str(Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.call(cmd)


def run_plumbing(args, rank, world, dist):
    """The multi-rank path without a GPU: every rank times a fixed host loop as its 'step' (the ranks' times differ),
    the job takes the slowest rank's time, and rank 0 prints the line with the whole job's value."""
    t0 = time.perf_counter()
    x = 0.0
    for i in range(20000 * (rank + 1)):
        x += i * 1e-9
    ms = (time.perf_counter() - t0) * 1e3
    ms_max = max_over_ranks(ms, dist, 'cpu')
    if rank == 0:
        print(json.dumps(dict(metric='rank plumbing (no GPU work)', value=job_value(world, 300.0, ms_max), unit='model days/s',
                              n_gpus=world, steps=1, warmup=0, ms_per_step=ms_max, rank_ms=ms, scaling='weak',
                              impl=args.impl)), flush=True)


def fp64_step_seconds(keys, warmup=3, steps=10):
    """Seconds per step of ONE member of each (level, layers) key alone on the plain FP64 core (its own batched graph):
    the sequential baseline of the ensemble and serving workloads."""
    import torch
    from isw import gpu
    from isw.batch import Batch
    from isw.ensemble import device_grids
    from isw.workload import Member
    gpu.set_precision('double')
    grids = device_grids(sorted({k[0] for k in keys}), 0)
    out = {}
    for level, layers in sorted(set(keys)):
        b = Batch(0)
        m = Member(grids[level], 0, ntracers=2, perturb=0.005, batch=b, kinds=('air',) if layers == 3 else ('air', 'ocean'),
                   init_device=torch.device('cuda:0'))
        for _ in range(warmup):
            b.step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            b.step()
        e1.record()
        torch.cuda.synchronize()
        out[(level, layers)] = e0.elapsed_time(e1) / steps / 1e3
        del m, b
    return out


def ensemble_result(steps, warmup, autotune_steps=3):
    """64 five-layer members (40 at level 5, 16 at level 6, 8 at level 7), seeds base + index, 0.5% perturbations, 2 FCT
    tracers, mixed precision, in one batch (one CUDA graph per step, tile layout by the autotuner); member-days/s
    against a sequential loop of the plain FP64 core over the same members."""
    import torch
    from isw.ensemble import Ensemble
    levels = [5] * 40 + [6] * 16 + [7] * 8
    t = time.time()
    ens = Ensemble.build(levels, seed=100, perturb=0.005, ntracers=2, precision='mixed', device=0)
    t_build = time.time() - t
    best, times = ens.batch.autotune(steps=autotune_steps)
    layout = ens.batch.info()
    for _ in range(warmup):
        ens.step()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record(st)
        for _ in range(steps):
            ens.step()
        e1.record(st)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    finite = all(bool(torch.isfinite(a).all()) for m in ens for a in m.state()) and ens.batch.status() == 0
    value = ens.member_days_per_step() / (ms / 1e3)
    launches = ens.members[0].launches() * steps
    footprint = ens.footprint()
    del ens
    base = fp64_step_seconds([(n, 5) for n in set(levels)])
    days = sum(cases_dt(n) for n in levels) / SECONDS_PER_DAY
    seq = days / sum(base[(n, 5)] for n in levels)
    return dict(metric='ensemble member-days/s: 64 five-layer members (40 x level 5, 16 x level 6, 8 x level 7), mixed form',
                value=value, unit='member-days/s', n_gpus=1, steps=steps, warmup=warmup, ms_per_step=ms,
                higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='f32 momentum, TRiSK operators and FCT corrections; f64 thickness, masses, budgets', data='synthetic',
                impl='isw',
                config=dict(workload='ensemble: 64 members, air 3 + ocean 2 layers, 2 tracers, 0.5% perturbations',
                            members=len(levels), l2='state far larger than L2 (no flush needed)'),
                layout=dict(stacks=layout['stacks'], tiles=layout, autotuned=best), device_bytes=footprint,
                sequential_fp64=dict(value=seq, unit='member-days/s', ms_per_member_step={f'level{k[0]}': v * 1e3 for k, v in base.items()},
                                     note='each member stepped alone on the plain FP64 core, one after another'),
                speedup_vs_sequential_fp64=value / seq, gpu_launches=launches, clocks=clk.summary(), finite=finite,
                build_s=t_build, autotune_ms={str(dict(k)): round(v, 4) for k, v in sorted(times.items(), key=lambda x: x[1])[:6]})


def cases_dt(level):
    from isw import cases
    return cases.stack_dt(level)


def run_ensemble(args):
    print(json.dumps(ensemble_result(args.steps, args.warmup)), flush=True)


def serving_result(requests, max_days, seed):
    """Seeded Poisson requests (rate 50 per second of the server's wall clock; level 4..7, horizon 1..max_days model days
    log-uniform, 3 or 5 layers), served with continuous batching in the mixed form under a 150 GB budget; p50/p99
    time-to-completion and member-days/s, against the plain FP64 core serving the same stream one request at a time."""
    from isw.serving import Server, poisson_requests, sequential_baseline
    reqs = poisson_requests(requests, 50.0, seed=seed, days=(1.0, max_days))
    srv = Server(0, budget_bytes=150e9, precision='mixed', ntracers=2)
    for n in sorted({r.level for r in reqs}):          # grids and the requests' initial states exist before the clock starts
        srv._grid(n)
    srv.prepare(reqs)
    with ClockSampler(0) as clk:
        results, stats = srv.run(reqs)
    del srv
    base = fp64_step_seconds({(r.level, r.layers) for r in reqs})

    def days_of(r):
        dt = cases_dt(r.level)
        n = max(1, int(math.ceil(r.days * SECONDS_PER_DAY / dt - 1e-9)))
        return n, n * dt / SECONDS_PER_DAY
    seq = sequential_baseline(reqs, base, days_of)
    return dict(metric='serving: p50/p99 time-to-completion (s) and member-days/s, Poisson stream of forecast requests, mixed form',
                value=stats['member_days_per_s'], unit='member-days/s', p50_s=stats['p50_s'], p99_s=stats['p99_s'],
                n_gpus=1, steps=stats['batched_steps'], warmup=0, higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='f32 momentum, TRiSK operators and FCT corrections; f64 thickness, masses, budgets', data='synthetic',
                impl='isw',
                config=dict(workload=f'serving: {requests} requests, Poisson rate 50/s (server wall clock), '
                                     f'level 4..7, horizon 1..{max_days:g} model days log-uniform, 3 or 5 layers, 2 tracers',
                            budget_bytes=150e9, seed=seed),
                stats=stats,
                sequential_fp64=dict(seq, note='the same stream served one request at a time (FIFO) on the plain FP64 core, '
                                               'service times from measured per-step times'),
                clocks=clk.summary())


def run_serving(args):
    print(json.dumps(serving_result(args.requests, args.max_days, args.seed)), flush=True)


def run_profile(args):
    """The workload without timing, for a profiler's launch list: --members members of the level-N workload in one form
    (--form) in one batch, the fast loop as --tiles says (auto, off, shared or packed), stepped --steps times."""
    import torch
    from isw import gpu
    from isw.ensemble import Ensemble
    g, _ = build_grid(args.level, 0)
    gpu.set_precision(args.form)
    try:
        grids = {args.level: gpu.DeviceGrid(g)}
    finally:
        gpu.set_precision('double')
    ens = Ensemble.build([args.level] * args.members, seed=0, perturb=0.01, ntracers=3, precision=args.form, grids=grids)
    if args.tiles == 'off':
        ens.batch.config(tiles=False)
    elif args.tiles != 'auto':
        ens.batch.config(tiles=True, layout=args.tiles)
    for _ in range(args.steps):
        ens.step()
    torch.cuda.synchronize()
    print(json.dumps(dict(workload='profile', form=args.form, level=args.level, members=args.members, steps=args.steps,
                          layout=ens.batch.info(), launches_per_step=ens.members[0].launches(), status=ens.batch.status())),
          flush=True)


def run_accuracy(args):
    """The mixed form against the plain FP64 form (error norms and mass drifts; no timing): the member over 10 model
    days at levels 6 (the benchmark member), 5 and 7 (the levels of the ensemble and serving workloads), the level-7
    Galewsky jet over 6 model days and Williamson 2 over 5 days at level 4."""
    from isw import accuracy
    out = dict(metric='mixed-form accuracy against the FP64 form', impl='isw', data='synthetic',
               member=accuracy.member(6, args.days_member), galewsky=accuracy.galewsky(7, args.days_galewsky),
               w2=accuracy.w2(4, 5.0),
               member_level5=accuracy.member(5, args.days_member), member_level7=accuracy.member(7, args.days_member))
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='isw', choices=('isw', 'reference'))
    ap.add_argument('--level', type=int, default=6)
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline leg')
    ap.add_argument('--percall', action='store_true', help='step call by call (one graph per stack) instead of the batched launch')
    ap.add_argument('--no-mixed', action='store_true', help='skip the mixed precision form')
    ap.add_argument('--no-configs', action='store_true', help='skip the level-7, ensemble and serving sub-measurements')
    ap.add_argument('--batched', type=int, default=8, help='members of the batched-core measurement (0: skip)')
    ap.add_argument('--workload', default='member', choices=('member', 'ensemble', 'serving', 'accuracy', 'profile'))
    ap.add_argument('--form', default='double', choices=('double', 'mixed'), help='profile: the precision form')
    ap.add_argument('--members', type=int, default=1, help='profile: members in the batch')
    ap.add_argument('--tiles', default='auto', choices=('auto', 'off', 'shared', 'packed'), help='profile: fast-loop layout')
    ap.add_argument('--days-member', type=float, default=10.0, help='accuracy: model days of the level-6 member')
    ap.add_argument('--days-galewsky', type=float, default=6.0, help='accuracy: model days of the Galewsky jet')
    ap.add_argument('--requests', type=int, default=48, help='serving: requests in the stream')
    ap.add_argument('--max-days', type=float, default=30.0, help='serving: longest horizon (model days)')
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--plumbing', action='store_true',
                    help='the rank plumbing alone on the CPU (gloo): ranks, barrier, max over ranks, the job value; no GPU work')
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.workload != 'member' and args.impl == 'isw':
        {'ensemble': run_ensemble, 'serving': run_serving, 'accuracy': run_accuracy, 'profile': run_profile}[args.workload](args)
        return

    if args.gpus > 1 and 'WORLD_SIZE' not in os.environ:
        sys.exit(spawn_ranks(args.gpus))         # one process per GPU, as torchrun would start them
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world != args.gpus:
        sys.exit(f'bench: {world} ranks for --gpus {args.gpus}')
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        if not args.plumbing:
            torch.cuda.set_device(local)
        dist.init_process_group('gloo' if args.plumbing else 'nccl', timeout=datetime.timedelta(seconds=600))
    if args.plumbing:
        run_plumbing(args, rank, world, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.impl == 'reference':
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    from isw import roofline
    from isw.batch import Batch
    from isw.gpu import DeviceGrid, set_precision
    from isw.workload import Member
    dev = torch.device(f'cuda:{local}')
    torch.cuda.set_device(dev)
    g, t_grid = build_grid(args.level, local)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    def make(precision, grid=None):
        set_precision(precision)
        try:
            dg = DeviceGrid(g if grid is None else grid, device=local)
            batch = None if args.percall else Batch(local)
            m = Member(dg, seed=rank, batch=batch)
        finally:
            set_precision('double')
        if batch is None:
            return m, None
        tuned, _ = batch.autotune(steps=3)       # tile layout by timing (the member's state is restored)
        return m, dict(batch.info(), autotuned=tuned)

    def timed(m):
        """Mean device ms per step over exactly args.steps steps (after the warm-up), max over ranks."""
        for _ in range(args.warmup):
            m.step()
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t_soak = time.time()                     # keep the GPU busy ~1 s so the clock samples cover load, then time
        while time.time() - t_soak < 1.0:
            for _ in range(20):
                m.step()
            torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()                        # the L2 holds no state from the previous step
            starts[k].record(stream)
            m.step()
            ends[k].record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t = sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / args.steps
        return max_over_ranks(t, dist, dev)

    member, layout = make('double')
    mixed, layout_m = (None, None) if args.no_mixed else make('mixed')
    with ClockSampler(local) as clk:
        ms = timed(member)
        ms_m = timed(mixed) if mixed is not None else None
    batched = None
    if mixed is not None and args.batched > 0 and not args.percall:
        # the batched core: args.batched members of the same workload (seeds rank * 1000 + i) in one batch, per form
        from isw.ensemble import Ensemble
        batched = dict(members=args.batched, level=args.level)
        for form in ('mixed', 'double'):
            set_precision(form)
            try:
                grids = {args.level: DeviceGrid(g, device=local)}
            finally:
                set_precision('double')
            ens = Ensemble.build([args.level] * args.batched, seed=rank * 1000, perturb=0.01, ntracers=3, precision=form,
                                 device=local, grids=grids)
            tuned, tried = ens.batch.autotune(steps=2)
            t_b = timed(ens)
            batched[form] = dict(value=world * ens.member_days_per_step() / (t_b / 1e3), unit='member-days/s',
                                 ms_per_step=t_b, layout=ens.batch.info(), autotuned=tuned,
                                 autotune_ms={str(dict(k)): round(v, 4) for k, v in sorted(tried.items(), key=lambda x: x[1])[:6]},
                                 finite=all(bool(torch.isfinite(a).all()) for m_ in ens for a in m_.state()),
                                 status=ens.batch.status())
            del ens

    finite = all(bool(torch.isfinite(a).all()) for a in member.state())
    status = [st for st in (member_status(member), member_status(mixed)) if st]   # a failed step voids the line
    if status:
        raise RuntimeError(f'bench: a timed step reported failure status {status}')
    dt = member.dt
    value = job_value(world, dt, ms)
    if batched is not None:
        batched['mixed_vs_fp64_member'] = batched['mixed']['value'] / value
        batched['mixed_vs_fp64_batched'] = batched['mixed']['value'] / batched['double']['value']

    # end to end through the public API with host buffers: H2D of the state, the step, D2H of the state, every step
    host = [torch.empty(a.shape, dtype=a.dtype, pin_memory=True) for a in member.state()]
    for hbuf, a in zip(host, member.state()):
        hbuf.copy_(a)
    torch.cuda.synchronize()
    e2e_steps = max(3, args.steps // 2)
    # A host caller's loop: every step copies its inputs in from pinned host memory and its results out to it. The
    # copies in run on one stream and the copies out on another, array by array, so the two directions of the link
    # overlap: array k of step n + 1 goes in as soon as array k of step n has come out (its host buffer is the input).
    # The step waits for all of its inputs; its results go out once it is done.
    state = member.state()
    c_in, c_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    out_ev = [torch.cuda.Event() for _ in state]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    c_in.wait_stream(stream)
    c_out.wait_stream(stream)
    for n in range(e2e_steps):
        with torch.cuda.stream(c_in):
            for k, (hbuf, a) in enumerate(zip(host, state)):
                if n > 0:
                    c_in.wait_event(out_ev[k])
                a.copy_(hbuf, non_blocking=True)
        stream.wait_stream(c_in)
        member.step()
        c_out.wait_stream(stream)
        with torch.cuda.stream(c_out):
            for k, (hbuf, a) in enumerate(zip(host, state)):
                hbuf.copy_(a, non_blocking=True)
                out_ev[k].record(c_out)
    stream.wait_stream(c_out)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, dist, dev)
    io_bytes = sum(a.numel() * a.element_size() for a in member.state())

    impl_bytes = 0
    for s in member.stacks:
        N, E, NV, nE2 = roofline.grid_sizes(g)
        impl_bytes += roofline.layers_step_bytes(N, E, NV, nE2, s.L, s.nfast, nu4=bool(s.core.nu4), vmix=bool(s.core.vmix))
        impl_bytes += roofline.transport_bytes(N, E, s.L, s.T)
    bytes_step = roofline.minimal_member_bytes(g.E, 'double')
    peak, peak_kind = peaks()
    achieved = bytes_step / (ms / 1e3) / 1e9
    traffic = None
    tf = ROOT / 'profiles' / 'traffic.json'
    if tf.exists():
        traffic = json.loads(tf.read_text()).get(f'level{args.level}_step_bytes')

    out = dict(metric=metric_name(args.level), value=value, unit='model days/s', n_gpus=world, steps=args.steps,
               warmup=args.warmup, ms_per_step=ms, higher_is_better=True, scaling='weak', vs_baseline=None, dtype='f64',
               data='synthetic', impl='isw',
               config=member_config(args, g, world),
               layout=dict(precision='fp64', tiles=layout,
                           launch='call by call' if args.percall else 'one CUDA graph per step (phase kernels + tiled fast loop)'),
               roofline=dict(bound='hbm', achieved=achieved, peak=peak, unit='GB/s', frac=achieved / peak, traffic=traffic,
                             peak_kind=peak_kind, algorithmic_bytes_per_step=bytes_step, unit_of_work='one member step',
                             bytes_model='minimal phase decomposition (compulsory traffic)',
                             implementation_bytes_per_step=impl_bytes),
               e2e=dict(value=job_value(world, dt, e2e_ms), unit='model days/s',
                        h2d_bytes_per_step=io_bytes, d2h_bytes_per_step=io_bytes),
               gpu_launches=member.launches() * args.steps, clocks=clk.summary(), finite=finite, grid_build_s=t_grid)
    if mixed is not None:
        vm = job_value(world, dt, ms_m)
        out['mixed'] = dict(value=vm, unit='model days/s', ms_per_step=ms_m, speedup_vs_fp64=vm / value, steps=args.steps,
                            dtype='f32 momentum, TRiSK operators and FCT corrections; f64 thickness, masses, budgets',
                            tiles=layout_m, finite=all(bool(torch.isfinite(a).all()) for a in mixed.state()),
                            gpu_launches=mixed.launches() * args.steps)
    if batched is not None:
        out['batched'] = batched

    if world == 1 and not args.no_configs and not args.percall:
        # the beyond-L2 member (level 7, both forms) and the ensemble and serving workloads, shortened to a few
        # timed steps and a short request stream so that the default run stays within a few minutes
        g7, _ = build_grid(7, local)
        l7 = dict(level=7, cells=int(g7.N), edges=int(g7.E))
        for form in ('double', 'mixed'):
            m7, lay7 = make(form, g7)
            t7 = timed(m7)
            l7[form] = dict(ms_per_step=t7, value=job_value(1, m7.dt, t7), unit='model days/s', layout=lay7,
                            finite=all(bool(torch.isfinite(a).all()) for a in m7.state()))
            if form == 'double':
                a7 = roofline.minimal_member_bytes(g7.E, 'double') / (t7 / 1e3) / 1e9
                l7[form]['roofline'] = dict(achieved=a7, peak=peak, unit='GB/s', frac=a7 / peak,
                                            algorithmic_bytes_per_step=roofline.minimal_member_bytes(g7.E, 'double'))
            del m7
        l7['mixed_vs_fp64'] = l7['mixed']['value'] / l7['double']['value']
        out['level7'] = l7
        keep = ('metric', 'value', 'unit', 'ms_per_step', 'steps', 'warmup', 'p50_s', 'p99_s', 'config', 'layout',
                'sequential_fp64', 'speedup_vs_sequential_fp64', 'device_bytes', 'finite', 'gpu_launches', 'stats',
                'autotune_ms')
        ens = ensemble_result(steps=5, warmup=3, autotune_steps=2)
        out['ensemble'] = {k: v for k, v in ens.items() if k in keep}
        srv = serving_result(requests=24, max_days=3.0, seed=args.seed)
        out['serving'] = {k: v for k, v in srv.items() if k in keep}
        out['serving']['note'] = 'a shortened stream (24 requests, horizons 1..3 model days); --workload serving runs the full one'

    if rank == 0 and world == 1 and not args.no_cpu:
        ensure_oracle()
        step, _ = cpu_member(g, 0, 'oracle')
        sec, n = time_cpu(step, budget_s=15.0, max_steps=50)
        out['cpu_baseline'] = dict(value=dt / SECONDS_PER_DAY / sec, unit='model days/s', cores=os.cpu_count() or 1, kind='port',
                                   sample=f'{n} full steps of the same member (the C oracle, OpenMP on all host threads)')
        # the single-process leg: the same kernels as whole-array NumPy operations, one process, no threads
        step, _ = cpu_member(g, 0, 'numpy')
        sec, n = time_cpu(step, budget_s=8.0, max_steps=5)
        out['cpu_baseline_numpy'] = dict(value=dt / SECONDS_PER_DAY / sec, unit='model days/s', cores=1, kind='port',
                                         sample=f'{n} full steps of the same member (the oracle kernels in NumPy, one process)')
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
