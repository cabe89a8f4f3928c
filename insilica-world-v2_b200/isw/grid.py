"""Host-side grid container with the reference's array names (reference ``src/insilica/grid/__init__.py:67-83``),
and the planet scaling of a cached Earth-sized grid (``grid/__init__.py:39-53``)."""
import numpy as np

R_PLANET = 6.371e6
OMEGA_REF = 2 * np.pi / 86400
GRAV = 9.80616
LENGTHS, AREAS = ('de', 'dist', 'edgeLen', 'le'), ('area', 'areaCell', 'areaV', 'kite', 'totalArea')


class Grid:
    """Attributes are the reference's array names (pos, nbr, eI, cellEdge, le, w, ...)."""

    def __init__(self, arrays):
        self._keys = sorted(arrays)
        for k, v in arrays.items():
            setattr(self, k, v[()] if isinstance(v, np.ndarray) and v.ndim == 0 else v)
        self.n, self.N, self.E, self.NV = int(self.n), int(self.N), int(self.E), int(self.NV)

    def arrays(self):
        return {k: getattr(self, k) for k in self._keys}

    def __repr__(self):
        return f'Grid(n={self.n}, N={self.N}, E={self.E}, NV={self.NV})'


def load(path):
    with np.load(path) as z:
        return Grid({k: z[k] for k in z.files if not k.startswith('sha_')})


def for_planet(g, radius=R_PLANET, omega=OMEGA_REF, grav=GRAV):
    """The grid on a planet of this radius and rotation: lengths and areas scaled, fV scaled by omega / Omega_ref."""
    if radius == R_PLANET and omega == OMEGA_REF and grav == GRAV:
        return g
    a, s = g.arrays(), radius / R_PLANET
    for k in LENGTHS:
        if k in a:
            a[k] = a[k] * s
    for k in AREAS:
        if k in a:
            a[k] = a[k] * s * s
    a['fV'] = a['fV'] * (omega / OMEGA_REF)
    a.update(radius=float(radius), omega=float(omega), grav=float(grav))
    return Grid(a)


MESH_KEYS = ('n', 'N', 'E', 'NV', 'pos', 'lat', 'lon', 'area', 'east', 'north', 'nbr', 'deg', 'dist', 'edgeLen', 'edgeDir',
             'corners', 'totalArea', 'lloydIters', 'lloydMoved', 'eI', 'eJ', 'eKi', 'eKj', 'perm', 'vPos', 'xm', 'cornerV',
             'cellEdge', 'cellSign', 'ev1', 'ev2', 'de', 'le', 'xe', 'ne', 'kite', 'areaCell', 'areaV', 'circ1', 'circ2', 'fV',
             'eoeStart', 'eoe', 'w', 'cellEdgeAsc', 'vEdge', 'vEdgeSign', 'vCell', 'vSlot')
LLOYD = {'converged': 200000, 'v1': 400}        # iteration caps; both stop at the 1e-11 rad tolerance (grid/__init__.py:28)


def build(n, order='hilbert', lloyd='converged', device=None, pos_v1=None):
    """Build level n with the C library (icosphere, Lloyd, geometry, renumbering, TRiSK tables; the reference's
    grid.make, grid/__init__.py:86-103). device: a CUDA device index for the Lloyd iterations, or 'cpu' (host cores);
    default: the GPU when one is present and n >= 5. pos_v1: smoothed positions in the icosphere's numbering (N, 3)
    to use instead of running Lloyd."""
    import ctypes
    from . import _lib
    if device is None:
        try:
            import torch
            device = torch.cuda.current_device() if (n >= 5 and torch.cuda.is_available()) else 'cpu'
        except ImportError:
            device = 'cpu'
    dev = -1 if device == 'cpu' else int(device)
    pv = None
    if pos_v1 is not None:
        pv = np.ascontiguousarray(pos_v1, dtype=np.float64)
        if pv.shape != (10 * 4 ** n + 2, 3):
            raise ValueError('build: pos_v1 must be (N, 3)')
    h = ctypes.c_void_p()
    _lib.check(_lib.isw_mesh_build(int(n), 0 if order == 'v1' else 1, LLOYD[lloyd], dev,
                                   _lib.host_ptr(pv) if pv is not None else None, ctypes.byref(h)))
    try:
        out = {}
        keys = MESH_KEYS if order != 'v1' else tuple(k for k in MESH_KEYS if k != 'perm')
        for k in keys:
            data, count, kind = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_int()
            _lib.check(_lib.isw_mesh_get(h, k.encode(), ctypes.byref(data), ctypes.byref(count), ctypes.byref(kind)))
            c, kd = count.value, kind.value
            if kd == 5:
                out[k] = int(ctypes.cast(data, ctypes.POINTER(ctypes.c_int64))[0])
                continue
            if kd == 6:
                out[k] = float(ctypes.cast(data, ctypes.POINTER(ctypes.c_double))[0])
                continue
            dt, width = {0: (np.float64, 1), 1: (np.int32, 1), 2: (np.int8, 1), 3: (np.uint8, 1), 4: (np.float64, 3)}[kd]
            nbytes = c * width * np.dtype(dt).itemsize
            a = np.frombuffer(ctypes.string_at(data, nbytes), dtype=dt).copy() if c else np.zeros(0, dt)
            out[k] = a.reshape(-1, 3) if width == 3 else a
    finally:
        _lib.isw_mesh_destroy(h)
    N = out['N']
    for k in ('nbr', 'cellEdge', 'cellSign', 'cellEdgeAsc', 'cornerV', 'dist', 'edgeLen', 'kite'):
        out[k] = out[k].reshape(N, 6)
    for k in ('corners', 'edgeDir'):
        out[k] = out[k].reshape(N, 6, 3)
    for k in ('vEdge', 'vEdgeSign', 'vCell', 'vSlot'):
        out[k] = out[k].reshape(-1, 3)
    out['order'], out['lloyd'] = order, lloyd
    return Grid(out)
