"""Batched persistent steps (the reference's Ensemble, src/insilica/ensemble.py, as one launch): stacks registered once
and advanced together, each RK3 step + receiving masses + FCT transport + M <- M1 of every stack in ONE cooperative
kernel launch per step. A stack's results are bit-identical to stepping it alone through Layers/Transport."""
import ctypes

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

    def add(self, core, h, u, Fm, tr=None, M=None, M1=None, tracers=(), dt=None, nfast=None):
        """Register a stack: its Layers `core` and state (h, u, Fm), and optionally its Transport `tr` with M, M1 and the
        tracers. Returns the slot. The arrays are borrowed until remove()."""
        L, N, E, dev = core.L, core.dg.N, core.dg.E, self.device
        ptrs = (ctypes.c_void_p * max(1, len(tracers)))(*[device_ptr(t, shape=(L, N), name='tracer', device=dev) for t in tracers])
        slot = ctypes.c_int()
        _lib.check(_lib.isw_batch_add(self._h, core._h, tr._h if tr is not None else None,
                                      device_ptr(h, shape=(L, N), name='h', device=dev), device_ptr(u, shape=(L, E), name='u', device=dev),
                                      device_ptr(Fm, shape=(L, E), name='Fm', device=dev),
                                      device_ptr(M, shape=(L, N), name='M', device=dev) if tr is not None else None,
                                      device_ptr(M1, shape=(L, N), name='M1', device=dev) if tr is not None else None,
                                      ptrs, len(tracers), float(dt), int(nfast), ctypes.byref(slot)))
        self._keep[slot.value] = (core, tr, h, u, Fm, M, M1, tuple(tracers))
        return slot.value

    def remove(self, slot):
        _lib.check(_lib.isw_batch_remove(self._h, int(slot)))
        self._keep.pop(slot, None)

    def config(self, tiles=True, tile_k=8):
        """The fast loop in shared-memory tiles exchanging every k <= tile_k sub-steps (the largest that fits), or
        grid-wide passes."""
        _lib.check(_lib.isw_batch_config(self._h, 1 if tiles else 0, int(tile_k)))

    def info(self):
        """(stacks, tiles, exchange interval k, tile shared memory bytes) of the current layout."""
        st, ti, k, sm = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        _lib.check(_lib.isw_batch_info(self._h, ctypes.byref(st), ctypes.byref(ti), ctypes.byref(k), ctypes.byref(sm)))
        return dict(stacks=st.value, tiles=ti.value, tile_k=k.value, smem=sm.value)

    def step(self, stream=None):
        _lib.check(_lib.isw_batch_step(self._h, stream_of(self.device, stream)))

    def status(self, reset=False, stream=None):
        """The device status word: 0, or ISW_ETIMEOUT (5) after a grid barrier's bounded wait ran out."""
        st = _lib.isw_batch_status(self._h, stream_of(self.device, stream), 1 if reset else 0)
        if st not in (_lib.ISW_OK, _lib.ISW_ETIMEOUT):
            _lib.check(st)
        return st

    def fault_test(self, timeout_s=0.05, stream=None):
        """One step in which a block never arrives at the first barrier: the others' bounded waits run out."""
        _lib.check(_lib.isw_batch_fault_test(self._h, int(timeout_s * 1e9), stream_of(self.device, stream)))
