"""Flux-corrected tracer transport on the isw CUDA core (reference src/insilica/transport.py).

Works on the mass-weighted tracer M psi given each edge's volume flux Fm (per step, eI -> eJ positive). order 1:
first-order upwind; order 3: 3rd-order fluxes in RK3 stages with Zalesak FCT against the upwind solution. Arrays are
layered: psi, M0, M1 (L, N); Fm (L, E). Every tracer goes through the same launches; nothing is allocated per step.
"""
import ctypes

from . import _lib
from .gpu import as_device_grid, device_ptr, stream_of

BETA = 0.25         # upwind weight of the 3rd-order flux (reference transport.py:15)


class Transport:
    def __init__(self, dg, layers=1, beta=BETA, tracers=1, precision=None):
        """The reference's constructor (transport.py:19). precision (this core's): 'double' or 'mixed' for this object
        (the form of the batched FCT passes); None takes the grid's form."""
        if precision not in (None, 'double', 'mixed'):
            raise ValueError(f'Transport: precision {precision!r}, want double or mixed')
        dg = as_device_grid(dg)         # the reference's own DeviceGrid is accepted too (its host Grid is used)
        self.dg, self.L, self.beta, self.K = dg, layers, beta, tracers
        h = ctypes.c_void_p()
        mixed = dg.mixed if precision is None else precision == 'mixed'
        prec = _lib.ISW_MIXED if mixed else _lib.ISW_FP64
        _lib.check(_lib.isw_transport_create(dg.handle, int(layers), float(beta), int(tracers), prec, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, '_h', None)
        destroy = getattr(_lib, 'isw_transport_destroy', None) if _lib is not None else None
        if h is not None and h.value and destroy is not None:      # (module globals are gone at interpreter exit)
            destroy(h)
            self._h = None

    def mass_after(self, M0, Fm, M1, stream=None):
        """M1 = M0 moved by Fm (what the cells hold after the step)."""
        L, N, E, dev = self.L, self.dg.N, self.dg.E, self.dg.device
        _lib.check(_lib.isw_transport_mass_after(self._h, device_ptr(M0, shape=(L, N), name='M0', device=dev),
                                                 device_ptr(Fm, shape=(L, E), name='Fm', device=dev),
                                                 device_ptr(M1, shape=(L, N), name='M1', device=dev), stream_of(dev, stream)))

    def step(self, M0, M1, Fm, psi, order=3, stream=None):
        return self.step_many(M0, M1, Fm, [psi], order, stream)[0]

    def step_many(self, M0, M1, Fm, tracers, order=3, stream=None):
        """Move each (L, N) tracer in `tracers` by the same mass fluxes, in place, in one set of launches."""
        n = len(tracers)
        assert n <= self.K
        L, N, E, dev = self.L, self.dg.N, self.dg.E, self.dg.device
        ptrs = (ctypes.c_void_p * n)(*[device_ptr(t, shape=(L, N), name='tracer', device=dev) for t in tracers])
        _lib.check(_lib.isw_transport_step_many(self._h, device_ptr(M0, shape=(L, N), name='M0', device=dev),
                                                device_ptr(M1, shape=(L, N), name='M1', device=dev),
                                                device_ptr(Fm, shape=(L, E), name='Fm', device=dev), ptrs, n, int(order),
                                                stream_of(dev, stream)))
        return tracers
