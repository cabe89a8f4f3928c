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
