"""Batched steps (the reference's Ensemble, src/insilica/ensemble.py, as one CUDA graph): stacks registered once and
advanced together, each RK3 step + receiving masses + FCT transport + M <- M1 of every stack in one graph launch per
step (one kernel per phase over all stacks, the barotropic sub-steps in shared-memory tiles). A stack's results are
bit-identical to stepping it alone through Layers/Transport. `autotune` picks the tile layout by timing the batch."""
import ctypes
import itertools

from . import _lib
from .gpu import device_ptr, stream_of


class Batch:
    def __init__(self, device=0):
        self.device = int(device)
        h = ctypes.c_void_p()
        _lib.check(_lib.isw_batch_create(self.device, ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def __del__(self):
        h = getattr(self, '_h', None)
        destroy = getattr(_lib, 'isw_batch_destroy', None) if _lib is not None else None
        if h is not None and h.value and destroy is not None:
            destroy(h)
            self._h = None

    def add(self, core, h, u, Fm, tr=None, M=None, M1=None, tracers=(), dt=None, nfast=None, theta=None):
        """Register a stack: its Layers `core` and state (h, u, Fm), and optionally its Transport `tr` with M, M1 and the
        tracers. Air layers also give their theta (L, N), updated in place as Layers.step(..., theta=) does. Returns the
        slot. The arrays are borrowed until remove()."""
        L, N, E, dev = core.L, core.dg.N, core.dg.E, self.device
        if bool(core.air) != (theta is not None):
            raise ValueError('Batch.add: theta is given exactly for air layers')
        ptrs = (ctypes.c_void_p * max(1, len(tracers)))(*[device_ptr(t, shape=(L, N), name='tracer', device=dev) for t in tracers])
        slot = ctypes.c_int()
        common = (device_ptr(h, shape=(L, N), name='h', device=dev), device_ptr(u, shape=(L, E), name='u', device=dev),
                  device_ptr(Fm, shape=(L, E), name='Fm', device=dev))
        tail = (device_ptr(M, shape=(L, N), name='M', device=dev) if tr is not None else None,
                device_ptr(M1, shape=(L, N), name='M1', device=dev) if tr is not None else None,
                ptrs, len(tracers), float(dt), int(nfast), ctypes.byref(slot))
        trh = tr._h if tr is not None else None
        if theta is None:
            _lib.check(_lib.isw_batch_add(self._h, core._h, trh, *common, *tail))
        else:
            _lib.check(_lib.isw_batch_add_air(self._h, core._h, trh, *common,
                                              device_ptr(theta, shape=(L, N), name='theta', device=dev), *tail))
        self._keep[slot.value] = (core, tr, h, u, Fm, M, M1, tuple(tracers) + ((theta,) if theta is not None else ()))
        return slot.value

    def remove(self, slot):
        _lib.check(_lib.isw_batch_remove(self._h, int(slot)))
        self._keep.pop(slot, None)

    LAYOUTS = {'auto': 0, 'shared': 1, 'packed': 2}

    LEVEL_MODES = {'batch': 0, 'untiled': 1, 'packed': 2}

    GRID_MODES = {'split': 0, 'persistent': 1}

    def config(self, tiles=True, tile_k=8, layout='auto', tile_cells=0, blocks_per_sm=0, persistent=False, levels=None,
               grid=None):
        """The fast loop in shared-memory tiles exchanging every k <= tile_k sub-steps (the largest that fits), or
        grid-wide passes; layout 'shared' (one cooperative launch, tiles in proportion to each stack's cells), 'packed'
        (tiles of about tile_cells owned cells, stacks packed into launches) or 'auto'; blocks_per_sm 1, 2 or 0 (auto).
        grid: how untiled stacks run their grid-wide sub-steps: 'split' (a cell launch and an edge launch per sub-step)
        or 'persistent' (one cooperative launch per stage, co-resident blocks meeting at a grid barrier after every pass);
        persistent=True is grid='persistent'. Results are the same bits either way.
        levels: {grid level: (mode, tile_cells, tile_k)} with mode 'untiled' or 'packed' (its own tile size and
        interval; 0 = the batch's): a layout per level."""
        if grid is None:
            grid = 'persistent' if persistent else 'split'
        if grid not in self.GRID_MODES:
            raise ValueError(f'batch.config: grid must be one of {sorted(self.GRID_MODES)}')
        self._config = dict(tiles=tiles, tile_k=tile_k, layout=layout, tile_cells=tile_cells, blocks_per_sm=blocks_per_sm,
                            grid=grid)
        if levels:
            self._config['levels'] = {int(k): tuple(v) for k, v in levels.items()}
        _lib.check(_lib.isw_batch_config(self._h, 1 if tiles else 0, int(tile_k), self.LAYOUTS[layout], int(tile_cells),
                                         int(blocks_per_sm)))
        _lib.check(_lib.isw_batch_grid_loop(self._h, self.GRID_MODES[grid]))
        for lv in set(getattr(self, '_levels', {})) | set((levels or {}).keys()):
            mode, cells, k = (levels or {}).get(lv, ('batch', 0, 0))
            _lib.check(_lib.isw_batch_level_layout(self._h, int(lv), self.LEVEL_MODES[mode], int(cells), int(k)))
        self._levels = dict(levels or {})

    @property
    def grid(self):
        """How untiled stacks run their grid-wide sub-steps: 'split' or 'persistent'."""
        return getattr(self, '_config', {}).get('grid', 'split')

    @property
    def persistent(self):
        return self.grid == 'persistent'

    def info(self):
        """The current layout: stacks, tiles, exchange interval k, the largest tile's shared memory (bytes), cooperative
        launches per stage (groups), tile blocks per SM, and how untiled stacks run their grid-wide sub-steps (grid;
        persistent: whether that is the persistent loop)."""
        v = [ctypes.c_int() for _ in range(3)] + [ctypes.c_longlong()] + [ctypes.c_int() for _ in range(2)]
        _lib.check(_lib.isw_batch_info(self._h, *[ctypes.byref(x) for x in v]))
        return dict(stacks=v[0].value, tiles=v[1].value, tile_k=v[2].value, smem=v[3].value, groups=v[4].value,
                    blocks_per_sm=v[5].value, grid=self.grid, persistent=self.persistent)

    def autotune(self, steps=5, candidates=None, stream=None, per_level=True):
        """Choose the fast-loop layout by timing: each candidate configuration (layout, blocks per SM, exchange interval,
        tile size; or no tiles, with the grid-wide sub-steps split or persistent) runs `steps` batched steps after
        one warm-up step, timed with CUDA events; then, for a batch of several grid levels (per_level), each level in turn tries its own
        layout (untiled, or packed with its own tile size and interval) from the best one. The fastest stays configured.
        Every registered array is restored afterwards, so the stacks' states are as before. Returns (best configuration,
        {configuration: ms per step})."""
        import torch
        arrays = []
        for keep in self._keep.values():
            core, tr, h, u, Fm, M, M1, tracers = keep
            arrays += [a for a in (h, u, Fm, M, M1) + tuple(tracers) if a is not None]
        saved = [a.clone() for a in arrays]
        if candidates is None:
            candidates = [dict(tiles=False, grid=g) for g in ('split', 'persistent')]
            for layout, bps, k in itertools.product(('shared', 'packed'), (1, 2), (2, 3, 4, 6, 8)):
                cells = (0,) if layout == 'shared' else ((256, 512) if bps == 2 else (512, 1024))
                for c in cells:
                    candidates.append(dict(tiles=True, layout=layout, blocks_per_sm=bps, tile_k=k, tile_cells=c))
        dev = torch.device(f'cuda:{self.device}')
        st = torch.cuda.current_stream(dev) if stream is None else stream

        def timed(cand):
            self.config(**cand)
            self.step(st)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(steps):
                self.step(st)
            e1.record(st)
            torch.cuda.synchronize(dev)
            return e0.elapsed_time(e1) / steps

        def key_of(cand):
            return tuple(sorted((k, tuple(sorted(v.items())) if isinstance(v, dict) else v) for k, v in cand.items()))
        times, seen, configs = {}, set(), {}
        for cand in candidates:
            self.config(**cand)
            lay = self.info()
            key = (lay['tiles'], lay['tile_k'], lay['groups'], lay['blocks_per_sm'], lay['smem'], lay['grid'])
            if key in seen:                       # the same layout as an earlier candidate
                continue
            seen.add(key)
            times[key_of(cand)] = timed(cand)
            configs[key_of(cand)] = cand
        best = configs[min(times, key=times.get)]
        levels = sorted({keep[0].dg.host.n for keep in self._keep.values()})
        if per_level and len(levels) > 1 and (not best.get('tiles', True) or best.get('layout') == 'packed'):
            # a layout per grid level: from the best batch-wide one, each level in turn tries untiled and packed tile
            # sizes and intervals with the others held (one pass of coordinate descent), keeping what is faster
            cur = dict(best, tiles=True, layout='packed')
            start = 'untiled' if not best.get('tiles', True) else 'batch'
            cur['levels'] = {lv: (start, 0, 0) for lv in levels}
            t_cur = times[key_of(best)]
            for lv in levels:
                for opt in (('untiled', 0, 0), ('packed', 512, 3), ('packed', 1024, 3), ('packed', 1024, 4),
                            ('packed', 2048, 4)):
                    if cur['levels'][lv] == opt:
                        continue
                    cand = dict(cur, levels={**cur['levels'], lv: opt})
                    t = timed(cand)
                    times[key_of(cand)] = t
                    if t < t_cur:
                        cur, t_cur = cand, t
            if t_cur < times[key_of(best)]:
                best = cur
        self.config(**best)
        for a, b in zip(arrays, saved):
            a.copy_(b)
        torch.cuda.synchronize(dev)
        return best, times

    def step(self, stream=None):
        _lib.check(_lib.isw_batch_step(self._h, stream_of(self.device, stream)))

    def pipeline(self, on=True):
        """Pipelined steps: each step runs its dynamics beside the previous step's transport (two branches of one
        graph); the registered masses and tracers lag by one step until flush(), after which the state is bit-identical
        to the plain order. add/remove/config flush first."""
        _lib.check(_lib.isw_batch_pipeline(self._h, 1 if on else 0))

    def flush(self, stream=None):
        """Complete a pipelined batch's last transport (a no-op otherwise)."""
        _lib.check(_lib.isw_batch_flush(self._h, stream_of(self.device, stream)))

    def status(self, reset=False, stream=None):
        """The device status word: 0, ISW_ETIMEOUT (5) after a grid barrier's bounded wait ran out, or ISW_ENOTFINITE (6)
        after a step left a NaN or Inf thickness. While it is set, step() raises IswError with that status; reset clears
        it (restore the state first)."""
        st = _lib.isw_batch_status(self._h, stream_of(self.device, stream), 1 if reset else 0)
        if st not in (_lib.ISW_OK, _lib.ISW_ETIMEOUT, _lib.ISW_ENOTFINITE):
            _lib.check(st)
        return st

    def fault_test(self, timeout_s=0.05, stream=None):
        """One step in which a block never arrives at the first barrier: the others' bounded waits run out."""
        _lib.check(_lib.isw_batch_fault_test(self._h, int(timeout_s * 1e9), stream_of(self.device, stream)))
