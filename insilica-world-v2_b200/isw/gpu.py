"""Device plumbing with the reference's interface (reference src/insilica/gpu.py): DeviceGrid, dsum, the precision switch.

Arrays on the device are torch CUDA tensors here (the reference's are CuPy arrays); any array exposing
``__cuda_array_interface__`` or ``__dlpack__`` is accepted wherever a device array is taken: only its pointer, dtype,
shape, contiguity and device are read, and the C library works on the caller's memory in place.
"""
import ctypes
import os
import weakref

import numpy as np
import torch

from . import _lib

# Precision forms (reference gpu.py:18-24): 'double' is the FP64 form that matches the reference bit for bit; 'mixed' does
# chosen arithmetic in FP32 with FP64 state and budgets.
PRECISION = os.environ.get('INSILICA_PRECISION', 'double')


def set_precision(p):
    global PRECISION
    assert p in ('mixed', 'double')
    PRECISION = p


def device_ptr(a, dtype=torch.float64, shape=None, name='array', device=None, numel=None):
    """Pointer of a C-contiguous device array of the given dtype and shape (or number of values; checked); None stays
    None."""
    if a is None:
        return None
    if not isinstance(a, torch.Tensor):
        if hasattr(a, '__cuda_array_interface__'):
            ai = a.__cuda_array_interface__
            want = {torch.float64: '<f8', torch.float32: '<f4'}[dtype]
            if ai['typestr'] != want:
                raise TypeError(f'{name}: dtype {ai["typestr"]}, want {want}')
            if ai.get('strides') is not None:
                shp, item = tuple(ai['shape']), np.dtype(want).itemsize
                cstr = tuple(int(item * np.prod(shp[i + 1:], dtype=np.int64)) for i in range(len(shp)))
                if tuple(ai['strides']) != cstr:
                    raise ValueError(f'{name}: not C-contiguous')
            if shape is not None and tuple(ai['shape']) != tuple(shape):
                raise ValueError(f'{name}: shape {tuple(ai["shape"])}, want {tuple(shape)}')
            if numel is not None and int(np.prod(ai['shape'], dtype=np.int64)) != numel:
                raise ValueError(f'{name}: {int(np.prod(ai["shape"], dtype=np.int64))} values, want {numel}')
            return ai['data'][0]
        a = torch.from_dlpack(a)
    if not a.is_cuda:
        raise TypeError(f'{name}: must be on a CUDA device')
    if a.dtype != dtype:
        raise TypeError(f'{name}: dtype {a.dtype}, want {dtype}')
    if not a.is_contiguous():
        raise ValueError(f'{name}: not contiguous')
    if shape is not None and tuple(a.shape) != tuple(shape):
        raise ValueError(f'{name}: shape {tuple(a.shape)}, want {tuple(shape)}')
    if numel is not None and a.numel() != numel:
        raise ValueError(f'{name}: {a.numel()} values, want {numel}')
    if device is not None and a.device.index != device:
        raise ValueError(f'{name}: on cuda:{a.device.index}, the grid is on cuda:{device}')
    return a.data_ptr()


def stream_of(device, stream=None):
    if stream is None:
        return torch.cuda.current_stream(device).cuda_stream
    return getattr(stream, 'cuda_stream', stream)


class DeviceGrid:
    """A Grid's arrays on the GPU (reference gpu.py:55-83): index tables int32/int8, geometry FP64, and the 3rd-order
    transport stencil (gpu.py:86-108), built and validated by the C library."""

    INT32 = ('eI', 'eJ', 'nbr', 'cellEdge', 'cellEdgeAsc', 'ev1', 'ev2', 'vEdge', 'vCell', 'eoeStart', 'eoe')
    INT8 = ('cellSign', 'vEdgeSign', 'vSlot')
    REALS = ('le', 'de', 'areaCell', 'areaV', 'fV', 'kite', 'w')

    def __init__(self, grid, dtype=np.float64, device=None):
        self.host = grid
        self.n, self.N, self.E, self.NV = int(grid.n), int(grid.N), int(grid.E), int(grid.NV)
        self.dtype = np.dtype(dtype)
        if self.dtype != np.float64:
            raise NotImplementedError('DeviceGrid: the state is FP64 (REAL=float is the reference speed probe only)')
        self.real = 'double'
        self.mixed = PRECISION == 'mixed'
        self.device = torch.cuda.current_device() if device is None else int(device)
        keep = {}
        for k in self.INT32:
            keep[k] = _lib.host_array(getattr(grid, k), np.int32)
        for k in self.INT8:
            keep[k] = _lib.host_array(getattr(grid, k), np.int8)
        for k in self.REALS + ('dist',):
            keep[k] = _lib.host_array(getattr(grid, k), np.float64)
        for k in ('deg', 'eKi', 'eKj'):
            keep[k] = _lib.host_array(getattr(grid, k), np.uint8)
        d = _lib.GridHost(n=self.n, N=self.N, E=self.E, NV=self.NV, **{k: _lib.host_ptr(v) for k, v in keep.items()})
        h = ctypes.c_void_p()
        _lib.check(_lib.isw_grid_create(ctypes.byref(d), self.device, ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def __getattr__(self, name):
        """The grid's tables as device arrays under the reference's attribute names (gpu.py:58-63: int32 / int8 index
        tables, FP64 geometry), made on first use, for callers that pass them to a kernel-table entry (world.py:317)."""
        kinds = {**{k: torch.int32 for k in self.INT32}, **{k: torch.int8 for k in self.INT8},
                 **{k: torch.float64 for k in self.REALS}}
        if name not in kinds or 'host' not in self.__dict__:
            raise AttributeError(name)
        cache = self.__dict__.setdefault('_dev', {})
        if name not in cache:
            cache[name] = torch.as_tensor(np.ascontiguousarray(getattr(self.host, name)), dtype=kinds[name],
                                          device=f'cuda:{self.device}')
        return cache[name]

    def __del__(self):
        h = getattr(self, '_h', None)
        destroy = getattr(_lib, 'isw_grid_destroy', None) if _lib is not None else None
        if h is not None and h.value and destroy is not None:      # (module globals are gone at interpreter exit)
            destroy(h)
            self._h = None


_FOREIGN = weakref.WeakKeyDictionary()


def as_device_grid(dg):
    """This core's DeviceGrid for `dg`: dg itself, or, for another device grid that carries the host Grid as `.host`
    (the reference's own DeviceGrid, whose `kernel()` the rest of the model keeps using to build its other kernels),
    an isw DeviceGrid built from that Grid once and cached with it, in the form its `mixed` attribute asks."""
    if isinstance(dg, DeviceGrid):
        return dg
    host = getattr(dg, 'host', None)
    if host is None:
        raise TypeError('expected an isw DeviceGrid or a device grid carrying its host Grid as .host')
    try:
        mine = _FOREIGN.get(dg)
    except TypeError:                         # an object without weak references: keep the grid on it
        mine = getattr(dg, '_isw_device_grid', None)
    if mine is None:
        global PRECISION
        prev = PRECISION
        PRECISION = 'mixed' if getattr(dg, 'mixed', False) else 'double'
        try:
            mine = DeviceGrid(host)
        finally:
            PRECISION = prev
        try:
            _FOREIGN[dg] = mine
        except TypeError:
            setattr(dg, '_isw_device_grid', mine)
    return mine


def dsum(x, y=None, stream=None):
    """Deterministic sum of x (or of x * y): the reference's fixed-order tree (gpu.py:111-126), bit-identical to it.
    Returns a Python float."""
    x = x if isinstance(x, torch.Tensor) else torch.from_dlpack(x)
    x = x.contiguous().reshape(-1)
    px = device_ptr(x, name='x')
    py = None
    if y is not None:
        y = y if isinstance(y, torch.Tensor) else torch.from_dlpack(y)
        y = y.contiguous().reshape(-1)
        if y.numel() != x.numel():
            raise ValueError('dsum: x and y differ in size')
        py = device_ptr(y, name='y')
    out = ctypes.c_double()
    with torch.cuda.device(x.device):          # the sum allocates and launches on the current device: make it x's
        _lib.check(_lib.isw_dsum(px, py, x.numel(), ctypes.byref(out), stream_of(x.device, stream)))
    return out.value
